// The C ABI (include/tomostar_cuda.h): context, seeds, ts_eik_solve, the self-test gate.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "eik_engine.h"
#include "host_geo.h"

using ts::host::Grid;

std::string& ts_thread_error() {
    thread_local std::string text;
    return text;
}

namespace {

int check_grid(ts_ctx* ctx, const ts_grid* g) {
    if (!g) return ctx->fail(TS_E_ARG, "grid is null");
    const char* bad = Grid::validate(*g);
    if (bad) return ctx->fail(TS_E_ARG, bad);
    return TS_OK;
}

}  // namespace

extern "C" {

int ts_cuda_create(int32_t device, ts_ctx** out) {
    if (!out) return TS_E_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return TS_E_NODEVICE;
    }
    if (device < 0 || device >= count) return TS_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return TS_E_CUDA;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TS_E_CUDA;
    if (!prop.cooperativeLaunch) return TS_E_NODEVICE;
    ts_ctx* ctx = new ts_ctx();
    ctx->device = device;
    ctx->name = prop.name;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->total_mem = prop.totalGlobalMem;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return TS_E_CUDA;
    }
    int* h = nullptr;
    if (cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped) != cudaSuccess) {
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return TS_E_CUDA;
    }
    *h = 0;
    ctx->cancel_host = h;
    if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->cancel_dev), h, 0) != cudaSuccess) {
        cudaFreeHost(h);
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return TS_E_CUDA;
    }
    {
        // The context's pool for stream-ordered allocations (without one they come from the device's
        // default pool, which releases freed memory at every synchronisation).
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if (cudaMemPoolCreate(&ctx->pool, &props) == cudaSuccess) {
            uint64_t keep = prop.totalGlobalMem / 4;
            cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            cudaGetLastError();
            ctx->pool = nullptr;
        }
    }
    *out = ctx;
    return TS_OK;
}

void ts_cuda_destroy(ts_ctx* ctx) {
    if (!ctx) return;
    {
        std::lock_guard<std::recursive_mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        ts::eik::models_free(ctx);
        ctx->drop_graph();
        for (auto& kv : ctx->bufs)
            if (kv.second.p) cudaFree(kv.second.p);
        for (auto& kv : ctx->pinned)
            if (kv.second.p) cudaFreeHost(kv.second.p);
        ctx->bufs.clear();
        if (ctx->cancel_host) cudaFreeHost(const_cast<int*>(ctx->cancel_host));
        if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
        cudaStreamDestroy(ctx->stream);
        // Allocations still held (rows not yet freed) keep the pool's memory until they are freed.
        if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    }
    delete ctx;
}

const char* ts_last_error(ts_ctx* ctx) { return ctx ? ctx->err.c_str() : ts_thread_error().c_str(); }

int ts_device_name(ts_ctx* ctx, char* buf, int32_t cap) {
    if (!ctx || !buf || cap <= 0) return TS_E_ARG;
    std::snprintf(buf, size_t(cap), "%s", ctx->name.c_str());
    return TS_OK;
}

const char* ts_last_stats(ts_ctx* ctx) { return ctx ? ctx->stats.c_str() : ""; }

void ts_set_cancel(ts_ctx* ctx, int32_t cancel) {
    if (ctx && ctx->cancel_host) *ctx->cancel_host = cancel ? 1 : 0;
}

int32_t ts_eik_suggest_batch(ts_ctx* ctx, int64_t nodes, int32_t precision) {
    if (!ctx || nodes <= 0) return 0;
    const int64_t real = 8;  // a double, or the FP32 precision's float pair (EikonalOpenCl.Real)
    (void)precision;
    size_t free_b = 0, total_b = 0;
    cudaSetDevice(ctx->device);
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    // One field plus its tile flags per batch member; the slowness once (EikonalOpenCl.cs:124-131).
    int64_t per_field = nodes * real + nodes / 256 + 1;
    int64_t budget = int64_t(double(free_b) * 0.8) - 2 * nodes * real;
    int64_t b = budget / per_field;
    return int32_t(std::max<int64_t>(0, std::min<int64_t>(b, 1024)));
}

int32_t ts_engine_shapes(int32_t* shapes, int32_t cap) {
    const auto& all = ts::eik::tile_shapes();
    for (size_t q = 0; q < all.size() && int32_t(q) < cap; q++) {
        shapes[4 * q] = all[q].id;
        shapes[4 * q + 1] = all[q].bx;
        shapes[4 * q + 2] = all[q].by;
        shapes[4 * q + 3] = all[q].bz;
    }
    return int32_t(all.size());
}

int ts_engine_set_scheduler(ts_ctx* ctx, int32_t scheduler) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (scheduler != 0 && scheduler != 1) return ctx->fail(TS_E_ARG, "scheduler must be 0 (lockstep) or 1 (flow)");
    ctx->scheduler = scheduler;
    ctx->drop_graph();
    return TS_OK;
}

int ts_engine_set_tile(ts_ctx* ctx, int32_t precision, int32_t shape_id) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    bool known = false;
    for (const auto& t : ts::eik::tile_shapes()) known |= t.id == shape_id;
    if (!known) return ctx->fail(TS_E_ARG, "unknown tile shape");
    if (precision == TS_PRECISION_F64) ctx->tile_f64 = shape_id;
    else if (precision == TS_PRECISION_F32) ctx->tile_f32 = shape_id;
    else return ctx->fail(TS_E_ARG, "precision must be 64 or 32");
    return TS_OK;
}

int32_t ts_point_source(const ts_grid* grid, const double* slowness, double lon, double lat, double depth_km,
                        double origin_time, double radius_cells, int32_t* idx_out, double* t_out, int32_t cap) {
    if (!grid || !slowness || Grid::validate(*grid)) return -1;
    Grid g(*grid);
    return ts::host::point_source(g, slowness, lon, lat, depth_km, origin_time, radius_cells, idx_out, t_out,
                                  std::max(0, cap));
}

int ts_eik_solve(ts_ctx* ctx, const ts_grid* grid, const double* slowness, int32_t n_fields,
                 const int32_t* seed_offsets, const int32_t* seed_index, const double* seed_time, int32_t precision,
                 int32_t mode, double tol, int32_t max_rounds, void* out, int32_t out_type, ts_eik_stats* stats) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    int rc = check_grid(ctx, grid);
    if (rc) return rc;
    if (!slowness || !seed_offsets || n_fields <= 0 || !out) return ctx->fail(TS_E_ARG, "null array or no fields");
    if (seed_offsets[n_fields] > 0 && (!seed_index || !seed_time)) return ctx->fail(TS_E_ARG, "null seed arrays");
    if (mode != TS_MODE_ENGINE && mode != TS_MODE_PLAIN && mode != TS_MODE_FAST) return ctx->fail(TS_E_ARG, "unknown mode");
    if (out_type != TS_OUT_F64 && out_type != TS_OUT_F32) return ctx->fail(TS_E_ARG, "unknown output type");
    if (!(tol >= 0)) return ctx->fail(TS_E_ARG, "tolerance must be >= 0");
    ts::eik::SolveIn in{};
    in.grid = grid;
    in.slowness = slowness;
    in.n_fields = n_fields;
    in.seed_offsets = seed_offsets;
    in.seed_index = seed_index;
    in.seed_time = seed_time;
    in.precision = precision;
    in.mode = mode;
    in.tol = tol;
    in.max_rounds = max_rounds;
    ts_eik_stats local{};
    return ts::eik::solve(ctx, in, out, out_type, stats ? stats : &local);
}

int ts_model_put(ts_ctx* ctx, const ts_grid* grid, const double* slowness, int32_t n_phases, int32_t precision,
                 int32_t* model_id) {
    if (!ctx || !model_id) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!grid || !slowness || n_phases <= 0) return ctx->fail(TS_E_ARG, "null grid or slowness");
    int id = 0;
    int rc = ts::eik::model_put(ctx, grid, slowness, n_phases, precision, &id);
    *model_id = id;
    return rc;
}

int ts_model_drop(ts_ctx* ctx, int32_t model_id) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return ts::eik::model_drop(ctx, model_id);
}

int ts_eik_solve_model(ts_ctx* ctx, int32_t model_id, int32_t phase, int32_t n_fields, const int32_t* seed_offsets,
                       const int32_t* seed_index, const double* seed_time, int32_t mode, double tol,
                       int32_t max_rounds, void* out, int32_t out_type, ts_eik_stats* stats) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    auto it = ctx->models.find(model_id);
    if (it == ctx->models.end()) return ctx->fail(TS_E_ARG, "unknown model");
    if (!seed_offsets || n_fields <= 0) return ctx->fail(TS_E_ARG, "no fields");
    if (seed_offsets[n_fields] > 0 && (!seed_index || !seed_time)) return ctx->fail(TS_E_ARG, "null seed arrays");
    if (mode != TS_MODE_ENGINE && mode != TS_MODE_PLAIN && mode != TS_MODE_FAST) return ctx->fail(TS_E_ARG, "unknown mode");
    if (out_type != TS_OUT_F64 && out_type != TS_OUT_F32 && out_type != TS_OUT_NONE)
        return ctx->fail(TS_E_ARG, "unknown output type");
    if (out_type != TS_OUT_NONE && !out) return ctx->fail(TS_E_ARG, "null output");
    if (!(tol >= 0)) return ctx->fail(TS_E_ARG, "tolerance must be >= 0");
    ts::eik::SolveIn in{};
    in.model_id = model_id;
    in.phase = phase;
    in.grid = &it->second->def;
    in.n_fields = n_fields;
    in.seed_offsets = seed_offsets;
    in.seed_index = seed_index;
    in.seed_time = seed_time;
    in.precision = it->second->precision;
    in.mode = mode;
    in.tol = tol;
    in.max_rounds = max_rounds;
    ts_eik_stats local{};
    return ts::eik::solve(ctx, in, out, out_type, stats ? stats : &local);
}

int ts_cuda_selftest(ts_ctx* ctx, int32_t precision, double* rel_err, char* msg, int32_t cap) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    // The reference's case (EikonalOpenCl.cs:348-358).
    ts_grid d{10, 12, 42, 44, -2, 120, 22, 20, 16, 0, nullptr};
    Grid g(d);
    std::vector<double> s(size_t(g.count()));
    for (int k = 0; k < g.nz; k++)
        for (int j = 0; j < g.ny; j++)
            for (int i = 0; i < g.nx; i++)
                s[g.index(i, j, k)] =
                    1 / (5.8 + 0.02 * g.dep[k] + 0.2 * std::sin(0.7 * i) + 0.15 * std::cos(0.5 * j));
    std::vector<int32_t> si(4096);
    std::vector<double> st(4096);
    int n = ts::host::point_source(g, s.data(), 10.37, 42.61, 8.3, 0, 3, si.data(), st.data(), 4096);
    si.resize(n);
    st.resize(n);
    std::vector<double> host = ts::host::relax_for_selftest(g, s.data(), si, st);
    std::vector<double> dev(host.size());
    int32_t off[2] = {0, n};
    int rc = ts_eik_solve(ctx, &d, s.data(), 1, off, si.data(), st.data(), precision, TS_MODE_ENGINE,
                          1e-7 /* SettleTolerance */, 0, dev.data(), TS_OUT_F64, nullptr);
    char text[256];
    double rel = INFINITY;
    if (rc) {
        std::snprintf(text, sizeof text, "%s", ctx->err.c_str());
    } else {
        double lo = INFINITY, hi = -INFINITY, worst = 0;
        bool unreached = false;
        for (size_t q = 0; q < host.size(); q++) {
            if (!std::isfinite(host[q])) continue;
            if (!std::isfinite(dev[q])) { unreached = true; break; }
            lo = std::min(lo, host[q]);
            hi = std::max(hi, host[q]);
            worst = std::max(worst, std::fabs(dev[q] - host[q]));
        }
        if (unreached) {
            std::snprintf(text, sizeof text, "device left a node unreached");
        } else {
            rel = worst / std::max(1e-12, hi - lo);
            std::snprintf(text, sizeof text, "max |dt| %.2E s over a %.2f s field (%.2E relative)", worst, hi - lo, rel);
        }
    }
    if (rel_err) *rel_err = rel;
    if (msg && cap > 0) std::snprintf(msg, size_t(cap), "%s", text);
    if (rc) return rc;
    if (!(rel <= 1e-6)) return ctx->fail(TS_E_SELFTEST, text);
    return TS_OK;
}

}  // extern "C"
