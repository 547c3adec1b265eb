// The serving engine: a resident request loop with continuous batching.
//
// Inversion iterations, L-curve sweeps, resolution tests and relocation each ask for travel-time
// fields (and rays on them) on grids of their own, at their own pace. A server keeps the velocity
// models on the device and runs one loop thread over a single engine: requests wait in a FIFO
// queue, are admitted while their device footprint (the fields' engine buffers and float32 tables)
// fits in the HBM budget, and every admitted field joins the next epoch of the engine — a
// cooperative launch of a few sweep rounds over all fields in flight, whatever their grid. Fields
// keep their state between epochs, so a request admitted while others are half-way is solved
// alongside them, and a field's result does not depend on what it shared the device with. When
// all fields of a request have settled, its float32 tables are made on the device (the .qttb
// rounding, TravelTimeTable.Write), its rays traced on them (RayKernels.Compute), the tables
// copied to the caller's buffer if it gave one, and its memory returned to the budget.
//
// The reference has no serving loop; its batch is EikonalOpenCl.TrySolve on one grid
// (Forward/EikonalOpenCl.cs:138-166) and rays are RayKernels.Compute (Tomography/RayKernels.cs:30-115).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ctx.h"
#include "eik_engine.h"
#include "host_geo.h"
#include "rays.h"
#include "ts_common.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct ServeRequest {
    int64_t id = 0;
    int model_id = 0, phase = 0, n_fields = 0, n_rays = 0;
    std::vector<std::vector<int32_t>> seed_idx;
    std::vector<std::vector<double>> seed_t;
    std::vector<double> origin;      // 3 per field
    std::vector<int32_t> ray_field;  // per ray
    std::vector<double> ray_event;   // 3 per ray
    ts_grid inv{};
    std::vector<double> inv_depth;
    bool has_inv = false;
    double step_km = 0;
    float* tables_out = nullptr;
    // state
    std::vector<ts::eik::EngineField> fields;
    void* block = nullptr;
    size_t bytes = 0;
    float* tables_dev = nullptr;
    int status = -1;  // -1 queued, 0 running, 1 done
    bool admitted = false;
    int code = TS_OK;
    std::string error;
    ts_rows* rows = nullptr;
    Clock::time_point t_submit, t_admit, t_done;
    int rounds[2] = {0, 0};
};

}  // namespace

struct ts_server {
    ts_ctx* ctx = nullptr;
    int precision = TS_PRECISION_F64;
    int mode = TS_MODE_FAST;
    int tile = 2;
    int rounds_per_epoch = 1;
    size_t budget = 0;
    size_t in_use = 0, peak_use = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<ServeRequest*> pending;
    std::vector<ServeRequest*> running;
    std::map<int64_t, ServeRequest*> all;
    std::thread loop;
    bool stop = false;
    int64_t next_id = 1;
    // What submit checks a request against, kept here so that submitting never waits for an epoch.
    struct ModelInfo {
        int n_phases;
        int64_t count;
        bool variable;
    };
    std::map<int, ModelInfo> model_info;
    // statistics
    int64_t epochs = 0, fields_done = 0, requests_done = 0, node_updates = 0;
    double device_ms = 0, epoch_ms = 0, complete_ms = 0;
    std::string err;
};

namespace {

using ts::eik::EngineField;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

ts_grid coarsened(const ts_grid& g) {
    ts_grid c = g;
    c.nx = (g.nx - 1) / 2 + 1;
    c.ny = (g.ny - 1) / 2 + 1;
    c.nz = (g.nz - 1) / 2 + 1;
    c.depth_km = nullptr;
    return c;
}

// Device bytes a request holds while in flight: its fields' engine buffers and float32 tables.
size_t footprint(const ts_ctx::Model& m, int tile, int precision, int n_fields) {
    const ts::eik::FieldLayout L = ts::eik::field_layout(*m.grid, tile, precision);
    const size_t per = (size_t(L.bytes(precision)) + 255) / 256 * 256 + (size_t(m.grid->count()) * 4 + 255) / 256 * 256;
    return per * size_t(n_fields);
}

void finish(ts_server* sv, ServeRequest* r, int code, const std::string& why) {
    r->code = code;
    r->error = why;
    r->status = 1;
    r->t_done = Clock::now();
}

// Admits queued requests in arrival order while their footprint fits in the budget. Called with
// sv->mu held; allocations are stream-ordered on the server's stream.
void admit(ts_server* sv) {
    while (!sv->pending.empty()) {
        ServeRequest* r = sv->pending.front();
        auto it = sv->ctx->models.find(r->model_id);
        if (it == sv->ctx->models.end()) {
            sv->pending.pop_front();
            finish(sv, r, TS_E_ARG, "unknown model");
            sv->cv_done.notify_all();
            continue;
        }
        const ts_ctx::Model& m = *it->second;
        const size_t need = footprint(m, sv->tile, sv->precision, r->n_fields);
        if (need > sv->budget) {
            sv->pending.pop_front();
            finish(sv, r, TS_E_CAPACITY, "request needs more device memory than the whole budget");
            sv->cv_done.notify_all();
            continue;
        }
        if (sv->in_use + need > sv->budget) break;  // head of the queue waits for memory
        void* block = nullptr;
        if (sv->ctx->alloc_async(&block, need, sv->ctx->stream) != cudaSuccess) {
            cudaGetLastError();
            break;  // the device is short of memory now: retry after the next epoch frees some
        }
        sv->pending.pop_front();
        r->block = block;
        r->bytes = need;
        sv->in_use += need;
        sv->peak_use = std::max(sv->peak_use, sv->in_use);
        const ts::eik::FieldLayout L = ts::eik::field_layout(*m.grid, sv->tile, sv->precision);
        const size_t fb = (size_t(L.bytes(sv->precision)) + 255) / 256 * 256;
        char* p = static_cast<char*>(block);  // the fields' buffers, then their float32 tables
        const size_t esz = 8;  // model slowness: a double, or the FP32 precision's float pair
        r->fields.resize(r->n_fields);
        for (int f = 0; f < r->n_fields; f++) {
            EngineField& ef = r->fields[f];
            ts::eik::engine_field_place(ef, L, sv->precision, p);
            p += fb;
            ef.slowness = static_cast<const char*>(m.slowness) + size_t(r->phase) * m.grid->count() * esz;
            ef.seed_idx = r->seed_idx[f];
            ef.seed_t = r->seed_t[f];
            ef.cap = std::max(32, (m.grid->nx + m.grid->ny + m.grid->nz) / 4);
            ef.initialized = false;
            ef.status = 0;
        }
        r->tables_dev = reinterpret_cast<float*>(p);
        r->status = 0;
        r->admitted = true;
        r->t_admit = Clock::now();
        sv->running.push_back(r);
    }
}

// Tables, rays and copies of the requests whose fields have all stopped, as one batch: the tables
// of every field, then the rays of all requests on one model traced together and cut into each
// request's rows, then the copies the callers asked for, then one synchronisation. codes/errors
// receive each request's outcome.
void complete_batch(ts_server* sv, const std::vector<ServeRequest*>& reqs, std::vector<int>& codes,
                    std::vector<std::string>& errors) {
    ts_ctx* ctx = sv->ctx;
    codes.assign(reqs.size(), TS_OK);
    errors.assign(reqs.size(), std::string());
    auto fail = [&](size_t k, int rc) {
        codes[k] = rc;
        errors[k] = ctx->err;
    };
    for (size_t k = 0; k < reqs.size(); k++) {
        ServeRequest* r = reqs[k];
        const ts_ctx::Model& m = *ctx->models.at(r->model_id);
        const ts::eik::FieldLayout L = ts::eik::field_layout(*m.grid, sv->tile, sv->precision);
        bool settled = true;
        for (auto& ef : r->fields) {
            r->rounds[0] = std::max(r->rounds[0], ef.rounds[0]);
            r->rounds[1] = std::max(r->rounds[1], ef.rounds[1]);
            settled = settled && ef.status == 1;
        }
        if (!settled) {
            fail(k, ctx->fail(TS_E_UNSETTLED, "sweeping not settled within the round cap"));
            continue;
        }
        for (int f = 0; f < r->n_fields && codes[k] == TS_OK; f++) {
            int rc = ts::eik::field_to_dense_f32_device(ctx, *m.grid, L, r->fields[f].T, sv->precision,
                                                        r->tables_dev + size_t(f) * m.grid->count(), ctx->stream);
            if (rc) fail(k, rc);
        }
    }
    // Rays: requests on one model with the default inversion grid and step form one trace.
    std::map<int, std::vector<size_t>> groups;
    std::vector<size_t> singles;
    for (size_t k = 0; k < reqs.size(); k++) {
        if (codes[k] != TS_OK || reqs[k]->n_rays == 0) continue;
        if (!reqs[k]->has_inv && !(reqs[k]->step_km > 0)) groups[reqs[k]->model_id].push_back(k);
        else singles.push_back(k);
    }
    for (auto& grp : groups) {
        const ts_ctx::Model& m = *ctx->models.at(grp.first);
        const int64_t n = m.grid->count();
        std::vector<const float*> tables;
        std::vector<double> origin, events;
        std::vector<int32_t> table_of;
        std::vector<int> row_begin{0};
        for (size_t k : grp.second) {
            ServeRequest* r = reqs[k];
            const int base = int(tables.size());
            for (int f = 0; f < r->n_fields; f++) tables.push_back(r->tables_dev + size_t(f) * n);
            origin.insert(origin.end(), r->origin.begin(), r->origin.end());
            for (int a = 0; a < r->n_rays; a++) table_of.push_back(base + r->ray_field[a]);
            events.insert(events.end(), r->ray_event.begin(), r->ray_event.end());
            row_begin.push_back(row_begin.back() + r->n_rays);
        }
        ts_grid invdef = coarsened(m.def);
        ts::host::Grid inv(invdef);
        const double step = 0.5 * std::min(m.grid->min_spacing_km(), inv.min_spacing_km());  // RayKernels.cs:62
        ts_rows* all = nullptr;
        ts::rays::RayStats rst;
        int rc = ts::rays::trace_on_device(ctx, *m.grid, tables, origin.data(), inv, int(table_of.size()),
                                           table_of.data(), events.data(), step, &all, &rst);
        std::vector<ts_rows*> parts;
        if (rc == TS_OK) rc = ts::rays::split_rows(ctx, all, row_begin, parts);
        if (all) ts::rays::free_rows(all);
        for (size_t q = 0; q < grp.second.size(); q++) {
            if (rc) fail(grp.second[q], rc);
            else reqs[grp.second[q]]->rows = parts[q];
        }
    }
    for (size_t k : singles) {
        ServeRequest* r = reqs[k];
        const ts_ctx::Model& m = *ctx->models.at(r->model_id);
        ts_grid invdef = r->has_inv ? r->inv : coarsened(m.def);
        if (r->has_inv && !r->inv_depth.empty()) invdef.depth_km = r->inv_depth.data();
        if (const char* bad = ts::host::Grid::validate(invdef)) {
            fail(k, ctx->fail(TS_E_ARG, bad));
            continue;
        }
        ts::host::Grid inv(invdef);
        double step = r->step_km > 0 ? r->step_km : 0.5 * std::min(m.grid->min_spacing_km(), inv.min_spacing_km());
        ts::rays::RayStats rst;
        int rc = ts::rays::trace_on_device(ctx, *m.grid, r->tables_dev, r->n_fields, r->origin.data(), inv, r->n_rays,
                                           r->ray_field.data(), r->ray_event.data(), step, &r->rows, &rst);
        if (rc) fail(k, rc);
    }
    for (size_t k = 0; k < reqs.size(); k++) {
        ServeRequest* r = reqs[k];
        if (codes[k] != TS_OK || !r->tables_out) continue;
        const int64_t n = ctx->models.at(r->model_id)->grid->count();
        cudaError_t e = cudaMemcpyAsync(r->tables_out, r->tables_dev, sizeof(float) * size_t(n) * r->n_fields,
                                        cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            codes[k] = TS_E_CUDA;
            errors[k] = cudaGetErrorString(e);
        }
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        for (size_t k = 0; k < reqs.size(); k++)
            if (codes[k] == TS_OK) {
                codes[k] = TS_E_CUDA;
                errors[k] = cudaGetErrorString(e);
            }
    }
}

void release(ts_server* sv, ServeRequest* r) {
    if (r->block) {
        cudaFreeAsync(r->block, sv->ctx->stream);
        r->block = nullptr;
        sv->in_use -= r->bytes;
    }
}

void serve_loop(ts_server* sv) {
    ts_ctx* ctx = sv->ctx;
    cudaSetDevice(ctx->device);
    const double wake_rel = sv->mode == TS_MODE_FAST ? TS_WAKE_REL : 0.0;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv_work.wait(lk, [&] { return sv->stop || !sv->pending.empty() || !sv->running.empty(); });
            if (sv->stop) break;
            {
                std::lock_guard<std::recursive_mutex> cl(ctx->mu);
                admit(sv);
            }
            if (sv->running.empty()) {
                // The queue head waits for memory the device cannot give yet: look again shortly.
                sv->cv_work.wait_for(lk, std::chrono::milliseconds(2));
                continue;
            }
        }
        std::lock_guard<std::recursive_mutex> cl(ctx->mu);
        // One epoch over every field in flight; grids are those of the models in use.
        std::vector<const ts::host::Grid*> grids;
        std::vector<const ts::host::Metric*> metrics;
        std::map<int, int> grid_of_model;
        std::vector<EngineField*> fl;
        for (ServeRequest* r : sv->running) {
            auto gm = grid_of_model.find(r->model_id);
            int gi;
            if (gm == grid_of_model.end()) {
                const ts_ctx::Model& m = *ctx->models.at(r->model_id);
                gi = int(grids.size());
                grids.push_back(m.grid);
                metrics.push_back(m.metric);
                grid_of_model[r->model_id] = gi;
            } else {
                gi = gm->second;
            }
            for (auto& ef : r->fields) {
                ef.grid = gi;
                if (ef.status == 0) fl.push_back(&ef);
            }
        }
        ts_eik_stats st{};
        int rc = TS_OK;
        const auto te0 = Clock::now();
        if (!fl.empty()) {
            rc = sv->precision == TS_PRECISION_F64
                     ? ts::eik::engine_epoch<double>(ctx, grids, metrics, fl, ts::kSettleTolerance, wake_rel, sv->tile,
                                                     sv->rounds_per_epoch, &st, ctx->stream)
                     : ts::eik::engine_epoch<ts::Pair>(ctx, grids, metrics, fl, ts::kSettleTolerance, wake_rel, sv->tile,
                                                    sv->rounds_per_epoch, &st, ctx->stream);
        }
        const auto te1 = Clock::now();
        std::vector<ServeRequest*> still, finished;
        for (ServeRequest* r : sv->running) {
            bool stopped = true;
            for (auto& ef : r->fields) stopped = stopped && ef.status != 0;
            if (rc != TS_OK || stopped) finished.push_back(r);
            else still.push_back(r);
        }
        std::vector<int> codes;
        std::vector<std::string> errors;
        if (rc != TS_OK) {
            codes.assign(finished.size(), rc);
            errors.assign(finished.size(), ctx->err);
        } else {
            complete_batch(sv, finished, codes, errors);
        }
        const auto te2 = Clock::now();
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->epochs++;
        sv->device_ms += st.kernel_ms;
        sv->epoch_ms += ms_between(te0, te1);
        sv->complete_ms += ms_between(te1, te2);
        sv->node_updates += st.node_updates;
        sv->running.swap(still);
        for (size_t k = 0; k < finished.size(); k++) {
            release(sv, finished[k]);
            finish(sv, finished[k], codes[k], errors[k]);
            sv->fields_done += finished[k]->n_fields;
            sv->requests_done++;
        }
        if (!finished.empty()) sv->cv_done.notify_all();
    }
    // Shutdown: every request still queued or in flight ends with an error.
    std::lock_guard<std::mutex> lk(sv->mu);
    std::lock_guard<std::recursive_mutex> cl(ctx->mu);
    for (ServeRequest* r : sv->running) {
        release(sv, r);
        finish(sv, r, TS_E_CANCELLED, "server stopped");
    }
    for (ServeRequest* r : sv->pending) finish(sv, r, TS_E_CANCELLED, "server stopped");
    sv->running.clear();
    sv->pending.clear();
    cudaStreamSynchronize(ctx->stream);
    sv->cv_done.notify_all();
}

}  // namespace

extern "C" {

int ts_serve_create(int32_t device, int32_t precision, int32_t mode, int32_t tile, int32_t scheduler,
                    double hbm_budget_bytes, int32_t rounds_per_epoch, ts_server** out) {
    if (!out) return TS_E_ARG;
    *out = nullptr;
    if (precision != TS_PRECISION_F64 && precision != TS_PRECISION_F32) return TS_E_ARG;
    if (mode != TS_MODE_ENGINE && mode != TS_MODE_FAST) return TS_E_ARG;
    if (!(hbm_budget_bytes > 0)) return TS_E_ARG;
    bool known = false;
    for (const auto& t : ts::eik::tile_shapes()) known |= t.id == tile;
    if (!known) return TS_E_ARG;
    if (scheduler != 0 && scheduler != 1) return TS_E_ARG;
    ts_ctx* ctx = nullptr;
    int rc = ts_cuda_create(device, &ctx);
    if (rc) return rc;
    ctx->scheduler = scheduler;
    // Memory freed by finished requests stays with the context's stream-ordered pool for the next ones.
    cudaMemPool_t pool = ctx->pool;
    if (pool || cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    auto* sv = new ts_server();
    sv->ctx = ctx;
    sv->precision = precision;
    sv->mode = mode;
    sv->tile = tile;
    sv->budget = size_t(hbm_budget_bytes);
    sv->rounds_per_epoch = rounds_per_epoch > 0 ? rounds_per_epoch : 1;
    sv->loop = std::thread(serve_loop, sv);
    *out = sv;
    return TS_OK;
}

void ts_serve_destroy(ts_server* sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    if (sv->loop.joinable()) sv->loop.join();
    for (auto& kv : sv->all) {
        if (kv.second->rows) ts_rows_free(kv.second->rows);
        delete kv.second;
    }
    sv->all.clear();
    ts_cuda_destroy(sv->ctx);
    delete sv;
}

const char* ts_serve_last_error(ts_server* sv) { return sv ? sv->err.c_str() : ""; }

int ts_serve_set_epoch_ms(ts_server* sv, double ms) {
    if (!sv || !(ms >= 0)) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> cl(sv->ctx->mu);
    sv->ctx->epoch_budget_ms = ms;
    return TS_OK;
}

int ts_serve_model_put(ts_server* sv, const ts_grid* grid, const double* slowness, int32_t n_phases, int32_t* model_id) {
    if (!sv || !grid || !slowness || !model_id || n_phases < 1) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> cl(sv->ctx->mu);
    cudaSetDevice(sv->ctx->device);
    int rc = ts::eik::model_put(sv->ctx, grid, slowness, n_phases, sv->precision, model_id);
    if (rc) {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->err = sv->ctx->err;
        return rc;
    }
    const ts_ctx::Model& m = *sv->ctx->models.at(*model_id);
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->model_info[*model_id] = ts_server::ModelInfo{m.n_phases, m.grid->count(), m.grid->variable};
    return TS_OK;
}

int ts_serve_submit(ts_server* sv, const ts_serve_request* q, int64_t* request_id) {
    if (!sv || !q || !request_id) return TS_E_ARG;
    if (q->n_fields < 1 || !q->seed_offsets || q->n_rays < 0) return TS_E_ARG;
    if (q->seed_offsets[q->n_fields] > 0 && (!q->seed_index || !q->seed_time)) return TS_E_ARG;
    if (q->n_rays > 0 && (!q->ray_field || !q->ray_event || !q->field_origin)) return TS_E_ARG;
    auto r = std::make_unique<ServeRequest>();
    r->model_id = q->model_id;
    r->phase = q->phase;
    r->n_fields = q->n_fields;
    r->n_rays = q->n_rays;
    const auto t_submit = Clock::now();
    int64_t n = 0;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        auto it = sv->model_info.find(q->model_id);
        if (it == sv->model_info.end()) {
            sv->err = "unknown model";
            return TS_E_ARG;
        }
        if (q->phase < 0 || q->phase >= it->second.n_phases) {
            sv->err = "phase out of range";
            return TS_E_ARG;
        }
        if (q->n_rays > 0 && it->second.variable) {
            sv->err = "rays need uniform grids";
            return TS_E_ARG;
        }
        n = it->second.count;
    }
    for (int f = 0; f < q->n_fields; f++) {
        std::map<int32_t, double> merged;  // as TrySolve takes seed sets (EikonalOpenCl.cs:147-163)
        for (int s = q->seed_offsets[f]; s < q->seed_offsets[f + 1]; s++) {
            if (uint32_t(q->seed_index[s]) >= uint64_t(n)) continue;
            auto it = merged.find(q->seed_index[s]);
            if (it == merged.end() || q->seed_time[s] < it->second) merged[q->seed_index[s]] = q->seed_time[s];
        }
        if (merged.empty()) {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->err = "no seed nodes for field " + std::to_string(f);
            return TS_E_NOSEEDS;
        }
        std::vector<int32_t> si;
        std::vector<double> st;
        for (auto& kv : merged) {
            si.push_back(kv.first);
            st.push_back(kv.second);
        }
        r->seed_idx.push_back(std::move(si));
        r->seed_t.push_back(std::move(st));
    }
    if (q->field_origin) r->origin.assign(q->field_origin, q->field_origin + 3 * size_t(q->n_fields));
    if (q->n_rays > 0) {
        for (int a = 0; a < q->n_rays; a++)
            if (q->ray_field[a] < 0 || q->ray_field[a] >= q->n_fields) {
                std::lock_guard<std::mutex> lk(sv->mu);
                sv->err = "ray_field out of range";
                return TS_E_ARG;
            }
        r->ray_field.assign(q->ray_field, q->ray_field + q->n_rays);
        r->ray_event.assign(q->ray_event, q->ray_event + 3 * size_t(q->n_rays));
    }
    if (q->inv) {
        r->has_inv = true;
        r->inv = *q->inv;
        if (q->inv->depth_km) {
            r->inv_depth.assign(q->inv->depth_km, q->inv->depth_km + q->inv->nz);
            r->inv.depth_km = nullptr;
        }
    }
    r->step_km = q->step_km;
    r->tables_out = q->tables_out;
    r->t_submit = t_submit;
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) return TS_E_CANCELLED;
    r->id = sv->next_id++;
    *request_id = r->id;
    ServeRequest* raw = r.release();
    sv->all[raw->id] = raw;
    sv->pending.push_back(raw);
    sv->cv_work.notify_all();
    return TS_OK;
}

int ts_serve_wait(ts_server* sv, int64_t request_id, double timeout_s, ts_serve_result* res) {
    if (!sv || !res) return TS_E_ARG;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->all.find(request_id);
    if (it == sv->all.end()) return TS_E_ARG;
    ServeRequest* r = it->second;
    auto ready = [&] { return r->status == 1; };
    if (timeout_s < 0) sv->cv_done.wait(lk, ready);
    else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) return TS_E_TIMEOUT;
    std::memset(res, 0, sizeof(*res));
    res->status = r->code;
    res->n_fields = r->n_fields;
    res->rounds[0] = r->rounds[0];
    res->rounds[1] = r->rounds[1];
    res->queue_ms = ms_between(r->t_submit, r->admitted ? r->t_admit : r->t_done);
    res->latency_ms = ms_between(r->t_submit, r->t_done);
    res->rows = r->rows;
    std::strncpy(res->error, r->error.c_str(), sizeof(res->error) - 1);
    sv->all.erase(it);
    delete r;  // the rows now belong to the caller
    return TS_OK;
}

int ts_serve_stats(ts_server* sv, ts_serve_stats_t* out) {
    if (!sv || !out) return TS_E_ARG;
    std::lock_guard<std::mutex> lk(sv->mu);
    out->epochs = sv->epochs;
    out->fields_done = sv->fields_done;
    out->requests_done = sv->requests_done;
    out->node_updates = sv->node_updates;
    out->device_ms = sv->device_ms;
    out->epoch_ms = sv->epoch_ms;
    out->complete_ms = sv->complete_ms;
    out->bytes_in_use = double(sv->in_use);
    out->peak_bytes = double(sv->peak_use);
    out->queued = int32_t(sv->pending.size());
    out->in_flight = int32_t(sv->running.size());
    return TS_OK;
}

}  // extern "C"
