// Host orchestration of the eikonal solvers: the plain per-plane path and the tiled engine, and
// ts_eik_solve (EikonalOpenCl.TrySolve, Forward/EikonalOpenCl.cs:138-343).
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "ctx.h"
#include "eik_engine.h"
#include "eik_kernels.cuh"
#include "host_geo.h"

namespace ts {
namespace eik {

__global__ void fill_u8_kernel(uint8_t* __restrict__ p, uint8_t v, int64_t n) {
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n; q += int64_t(gridDim.x) * blockDim.x) p[q] = v;
}

template <typename From, typename To>
__global__ void convert_kernel(const From* __restrict__ a, To* __restrict__ b, int64_t n) {
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n; q += int64_t(gridDim.x) * blockDim.x)
        b[q] = To(a[q]);
}

static int fill_blocks(int64_t n) { return int(std::min<int64_t>((n + 255) / 256, 148 * 16)); }

// Seeds of one field, as TrySolve prepares them (EikonalOpenCl.cs:147-163): out-of-range nodes
// dropped, duplicates merged to the smallest time, ascending node order.
static void merge_seeds(const int32_t* idx, const double* t, int count, int64_t n, std::vector<int32_t>& out_idx,
                        std::vector<double>& out_t) {
    std::map<int32_t, double> m;
    for (int q = 0; q < count; q++) {
        if (uint32_t(idx[q]) >= uint64_t(n)) continue;
        auto it = m.find(idx[q]);
        if (it == m.end() || t[q] < it->second) m[idx[q]] = t[q];
    }
    out_idx.clear();
    out_t.clear();
    for (auto& kv : m) {
        out_idx.push_back(kv.first);
        out_t.push_back(kv.second);
    }
}

template <typename Real>
static int upload_real(ts_ctx* ctx, const std::string& key, const double* src, size_t count, Real** dst,
                       const float* src32 = nullptr) {
    std::vector<Real> tmp(count);
    for (size_t q = 0; q < count; q++) tmp[q] = src32 ? Real(weight_of<Real>(src[q], src32[q])) : Real(src[q]);
    TS_BUF(ctx, d, Real, key, count);
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d, tmp.data(), count * sizeof(Real), cudaMemcpyHostToDevice, ctx->stream));
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *dst = d;
    return TS_OK;
}

// ---- plain path ------------------------------------------------------------------------------------

// One field at a time, one launch per diagonal plane, the host reading the "changed" flag after
// every round (EikonalOpenCl.cs:196-270). The baseline the engine is measured against.
template <typename Real>
static int plain_solve(ts_ctx* ctx, const host::Grid& g, const host::Metric& m, const Real* slow_d, Real* T,
                       const std::vector<int32_t>& sidx, const std::vector<double>& st, double tol, int cap,
                       int rounds_out[2], ts_eik_stats* stats) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t n = g.count();
    Real *wx, *wy, *zc = nullptr;
    int rc;
    if ((rc = upload_real<Real>(ctx, "plain.wx", m.wx.data(), m.wx.size(), &wx, m.wx32.data()))) return rc;
    if ((rc = upload_real<Real>(ctx, "plain.wy", m.wy.data(), m.wy.size(), &wy, m.wy32.data()))) return rc;
    if (g.variable && (rc = upload_real<Real>(ctx, "plain.zc", m.zc.data(), m.zc.size(), &zc))) return rc;
    TS_BUF(ctx, fixed, uint8_t, "plain.fixed", n);
    TS_BUF(ctx, dirty, uint8_t, "plain.dirty", n);
    TS_BUF(ctx, changed, int, "plain.changed", 2);
    TS_BUF(ctx, updates, unsigned long long, "plain.updates", 1);
    TS_BUF(ctx, at, int64_t, "plain.seed_at", std::max<size_t>(1, sidx.size()));
    TS_BUF(ctx, tv, double, "plain.seed_t", std::max<size_t>(1, sidx.size()));
    std::vector<int64_t> at_h(sidx.begin(), sidx.end());
    cudaStream_t s = ctx->stream;
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(at, at_h.data(), at_h.size() * 8, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(tv, st.data(), st.size() * 8, cudaMemcpyHostToDevice, s));
    fill_kernel<Real><<<fill_blocks(n), 256, 0, s>>>(T, real_inf<Real>(), n);
    fill_u8_kernel<<<fill_blocks(n), 256, 0, s>>>(fixed, 0, n);
    TS_CUDA_TRY(ctx, cudaMemsetAsync(updates, 0, 8, s));
    seed_kernel<Real><<<(int(sidx.size()) + 127) / 128, 128, 0, s>>>(T, fixed, at, tv, int(sidx.size()));
    TS_CUDA_TRY(ctx, cudaGetLastError());
    const int planes = nx + ny + nz - 2;
    const Real wz1 = Real(weight_of<Real>(m.wz1, m.wz1_32)), wz2 = Real(weight_of<Real>(m.wz2, m.wz2_32));
    int launches = 0;
    struct Ev {  // events bracketing each round's plane launches
        cudaEvent_t e;
        Ev() { cudaEventCreate(&e); }
        ~Ev() { cudaEventDestroy(e); }
    } ev0, ev1;
    cudaEvent_t k0 = ev0.e, k1 = ev1.e;
    for (int phase = 0; phase < 2; phase++) {
        fill_u8_kernel<<<fill_blocks(n), 256, 0, s>>>(dirty, 1, n);
        bool settled = false;
        for (int round = 0; round < cap && !settled; round++) {
            if (ctx->cancel_host && *ctx->cancel_host) return ctx->fail(TS_E_CANCELLED, "cancelled");
            TS_CUDA_TRY(ctx, cudaMemsetAsync(changed, 0, sizeof(int), s));
            cudaEventRecord(k0, s);
            for (int dir = 0; dir < 8; dir++) {
                for (int p = 0; p < planes; p++) {
                    int i0 = std::max(0, p - (ny - 1) - (nz - 1)), i1 = std::min(nx - 1, p);
                    int k0 = std::max(0, p - (nx - 1) - (ny - 1)), k1 = std::min(nz - 1, p);
                    dim3 grid((i1 - i0 + 1 + 127) / 128, k1 - k0 + 1);
                    if (g.variable)
                        plain_sweep_kernel<Real, true><<<grid, 128, 0, s>>>(T, slow_d, fixed, dirty, wx, wy,
                                                                              wz1, wz2, zc, nx, ny, nz, phase,
                                                                              changed, dir, p, Real(tol), updates);
                    else
                        plain_sweep_kernel<Real, false><<<grid, 128, 0, s>>>(T, slow_d, fixed, dirty, wx, wy,
                                                                               wz1, wz2, zc, nx, ny, nz, phase,
                                                                               changed, dir, p, Real(tol), updates);
                    launches++;
                }
            }
            cudaEventRecord(k1, s);
            TS_CUDA_TRY(ctx, cudaGetLastError());
            int ch = 0;
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(&ch, changed, sizeof(int), cudaMemcpyDeviceToHost, s));
            TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
            float kms = 0;
            cudaEventElapsedTime(&kms, k0, k1);
            if (stats) stats->kernel_ms += kms;
            rounds_out[phase] = round + 1;
            settled = ch == 0;
        }
        if (!settled) {
            return ctx->fail(TS_E_UNSETTLED, "sweeping not settled after " + std::to_string(cap) + " rounds");
        }
    }
    unsigned long long up = 0;
    TS_CUDA_TRY(ctx, cudaMemcpy(&up, updates, 8, cudaMemcpyDeviceToHost));
    if (stats) {
        stats->node_updates += int64_t(up);
        stats->tile_visits += launches;
        stats->launches += launches;
    }
    return TS_OK;
}

// ---- resident models -----------------------------------------------------------------------------------

}  // namespace eik
}  // namespace ts

namespace ts {
namespace eik {

int model_put(ts_ctx* ctx, const ts_grid* grid, const double* slowness, int n_phases, int precision, int* id) {
    if (const char* bad = host::Grid::validate(*grid)) return ctx->fail(TS_E_ARG, bad);
    if (precision != TS_PRECISION_F64 && precision != TS_PRECISION_F32) return ctx->fail(TS_E_ARG, "precision");
    auto* m = new ts_ctx::Model();
    m->def = *grid;
    if (grid->depth_km) {
        m->depth.assign(grid->depth_km, grid->depth_km + grid->nz);
        m->def.depth_km = m->depth.data();
    }
    m->grid = new host::Grid(m->def);
    m->metric = new host::Metric(*m->grid);
    m->precision = precision;
    m->n_phases = n_phases;
    const size_t count = size_t(m->grid->count()) * n_phases;
    const size_t esz = 8;  // a double, or the FP32 precision's float pair (hi = the float slowness)
    if (cudaMalloc(&m->slowness, count * esz) != cudaSuccess) {
        cudaGetLastError();
        m->slowness = nullptr;
        delete m;
        return ctx->fail(TS_E_NOMEM, "model slowness");
    }
    int rc = TS_OK;
    if (precision == TS_PRECISION_F64) {
        if (cudaMemcpy(m->slowness, slowness, count * 8, cudaMemcpyHostToDevice) != cudaSuccess) rc = TS_E_CUDA;
    } else {
        std::vector<Pair> tmp(count);
        for (size_t q = 0; q < count; q++) tmp[q] = Pair(slowness[q]);
        if (cudaMemcpy(m->slowness, tmp.data(), count * sizeof(Pair), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = TS_E_CUDA;
    }
    if (rc) {
        delete m;
        return ctx->fail(rc, "model upload");
    }
    *id = ctx->next_model++;
    ctx->models[*id] = m;
    return TS_OK;
}

int model_drop(ts_ctx* ctx, int id) {
    auto it = ctx->models.find(id);
    if (it == ctx->models.end()) return ctx->fail(TS_E_ARG, "unknown model");
    delete it->second;
    ctx->models.erase(it);
    return TS_OK;
}

void models_free(ts_ctx* ctx) {
    for (auto& kv : ctx->models) delete kv.second;
    ctx->models.clear();
}

// ---- C-ABI front end ---------------------------------------------------------------------------------

template <typename Real>
static int solve_impl(ts_ctx* ctx, const SolveIn& in, void* out, int out_type, ts_eik_stats* stats) {
    ts_ctx::Model* model = nullptr;
    if (in.model_id > 0) {
        auto it = ctx->models.find(in.model_id);
        if (it == ctx->models.end()) return ctx->fail(TS_E_ARG, "unknown model");
        model = it->second;
        if (in.phase < 0 || in.phase >= model->n_phases) return ctx->fail(TS_E_ARG, "phase out of range");
    } else {
        const char* bad = host::Grid::validate(*in.grid);
        if (bad) return ctx->fail(TS_E_ARG, bad);
    }
    std::unique_ptr<host::Grid> own_g(model ? nullptr : new host::Grid(*in.grid));
    std::unique_ptr<host::Metric> own_m(model ? nullptr : new host::Metric(*own_g));
    const host::Grid& g = model ? *model->grid : *own_g;
    const host::Metric& m = model ? *model->metric : *own_m;
    const int64_t n = g.count();
    const int nf = in.n_fields;
    // Seeds of every field.
    std::vector<std::vector<int32_t>> sidx(nf);
    std::vector<std::vector<double>> st(nf);
    size_t total_seeds = 0;
    for (int f = 0; f < nf; f++) {
        int b = in.seed_offsets[f], e = in.seed_offsets[f + 1];
        if (e < b) return ctx->fail(TS_E_ARG, "seed offsets must not decrease");
        merge_seeds(in.seed_index + b, in.seed_time + b, e - b, n, sidx[f], st[f]);
        total_seeds += sidx[f].size();
    }
    if (total_seeds == 0) return ctx->fail(TS_E_NOSEEDS, "no seed nodes");
    for (int f = 0; f < nf; f++)
        if (sidx[f].empty()) return ctx->fail(TS_E_NOSEEDS, "no seed nodes for field " + std::to_string(f));
    // Slowness on the device in the solve's precision (the float kernel never meets a double).
    Real* slow_d;
    int rc = TS_OK;
    if (model) slow_d = static_cast<Real*>(model->slowness) + size_t(n) * in.phase;
    else if ((rc = upload_real<Real>(ctx, "solve.slowness", in.slowness, size_t(n), &slow_d))) return rc;
    const int cap = in.max_rounds > 0 ? in.max_rounds : std::max(32, (g.nx + g.ny + g.nz) / 4);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    int rounds_max[2] = {0, 0};
    EngineJob job;
    Real* T = nullptr;
    // Many fields into page-locked host memory: the copies of the first half overlap the second half's
    // solve (engine_run_to_host).
    bool pipelined = false;
    if (in.mode != TS_MODE_PLAIN && out_type != TS_OUT_NONE && out && nf >= 64 && !ctx->use_graph) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, out) == cudaSuccess) pipelined = at.type == cudaMemoryTypeHost;
        cudaGetLastError();
    }
    if (in.mode == TS_MODE_PLAIN) {
        T = static_cast<Real*>(ctx->buf("solve.fields", sizeof(Real) * size_t(nf) * n));
        if (!T) return TS_E_NOMEM;
        for (int f = 0; f < nf && rc == TS_OK; f++) {
            int r[2] = {0, 0};
            rc = plain_solve<Real>(ctx, g, m, slow_d, T + size_t(f) * n, sidx[f], st[f], in.tol, cap, r, stats);
            rounds_max[0] = std::max(rounds_max[0], r[0]);
            rounds_max[1] = std::max(rounds_max[1], r[1]);
        }
    } else {
        job.grids.push_back(&g);
        job.metrics.push_back(&m);
        job.tol = in.tol;
        job.wake_rel = in.mode == TS_MODE_FAST ? TS_WAKE_REL : 0.0;
        job.tile = is_f64<Real>() ? ctx->tile_f64 : ctx->tile_f32;
        for (int f = 0; f < nf; f++) {
            EngineField ef;
            ef.grid = 0;
            ef.slowness = slow_d;
            ef.seed_idx = std::move(sidx[f]);
            ef.seed_t = std::move(st[f]);
            ef.cap = cap;
            job.fields.push_back(ef);
        }
        rc = pipelined ? engine_run_to_host<Real>(ctx, job, out, out_type, stats) : engine_run<Real>(ctx, job, stats);
        for (auto& ef : job.fields) {
            rounds_max[0] = std::max(rounds_max[0], ef.rounds[0]);
            rounds_max[1] = std::max(rounds_max[1], ef.rounds[1]);
        }
        if (rc == TS_OK) {
            for (auto& ef : job.fields)
                if (ef.status != 1) {
                    rc = ctx->fail(TS_E_UNSETTLED, "sweeping not settled after " + std::to_string(cap) + " rounds");
                    break;
                }
        }
    }
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        stats->rounds[0] = rounds_max[0];
        stats->rounds[1] = rounds_max[1];
        stats->device_ms = ms;
    }
    ctx->stats = std::to_string(rounds_max[0]) + "+" + std::to_string(rounds_max[1]) + " rounds of 8 sweeps";
    if (rc) return rc;
    const int precision = precision_of<Real>();
    if (out_type == TS_OUT_NONE) return TS_OK;  // the fields stay on the device
    if (in.mode == TS_MODE_PLAIN) return copy_fields_out(ctx, T, precision, int64_t(nf) * n, out, out_type);
    if (pipelined) return TS_OK;  // already on the host
    return fields_to_dense_host(ctx, job, precision, out, out_type);
}

int solve(ts_ctx* ctx, const SolveIn& in, void* out, int out_type, ts_eik_stats* stats) {
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (in.precision == TS_PRECISION_F64) return solve_impl<double>(ctx, in, out, out_type, stats);
    if (in.precision == TS_PRECISION_F32) return solve_impl<Pair>(ctx, in, out, out_type, stats);
    return ctx->fail(TS_E_ARG, "precision must be 64 or 32");
}

// Device fields (precision) to host out (out_type), converted on the device in slabs.
int copy_fields_out(ts_ctx* ctx, const void* fields_dev, int precision, int64_t count, void* out, int out_type) {
    const bool src64 = precision == TS_PRECISION_F64;
    const bool dst64 = out_type == TS_OUT_F64;
    const size_t esz = dst64 ? 8 : 4;
    if (src64 && dst64) {
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(out, fields_dev, size_t(count) * esz, cudaMemcpyDeviceToHost, ctx->stream));
        TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        return TS_OK;
    }
    const int64_t slab = int64_t(32) << 20;  // elements per slab
    void* stage = ctx->buf("out.stage", size_t(std::min(count, slab)) * esz);
    if (!stage) return TS_E_NOMEM;
    for (int64_t o = 0; o < count; o += slab) {
        int64_t len = std::min(slab, count - o);
        if (src64)
            convert_kernel<double, float><<<fill_blocks(len), 256, 0, ctx->stream>>>(
                static_cast<const double*>(fields_dev) + o, static_cast<float*>(stage), len);
        else if (dst64)
            convert_kernel<Pair, double><<<fill_blocks(len), 256, 0, ctx->stream>>>(
                static_cast<const Pair*>(fields_dev) + o, static_cast<double*>(stage), len);
        else
            convert_kernel<Pair, float><<<fill_blocks(len), 256, 0, ctx->stream>>>(
                static_cast<const Pair*>(fields_dev) + o, static_cast<float*>(stage), len);
        TS_CUDA_TRY(ctx, cudaGetLastError());
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(static_cast<char*>(out) + o * esz, stage, size_t(len) * esz,
                                         cudaMemcpyDeviceToHost, ctx->stream));
    }
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return TS_OK;
}

}  // namespace eik
}  // namespace ts
