// Batches of fields on grids of uneven size in one engine launch, the engine's CUDA-graph switch and
// its tile-shape autotuner. The reference batches only fields sharing one grid and one slowness
// (EikonalOpenCl.TrySolve, Forward/EikonalOpenCl.cs:138-166); these entry points extend that batch.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <vector>

#include "ctx.h"
#include "eik_engine.h"
#include "host_geo.h"

namespace ts {
namespace eik {

template <typename Real>
static int solve_multi_impl(ts_ctx* ctx, int n_grids, const ts_grid* grids, const double* const* slowness,
                            int n_fields, const int32_t* field_grid, const int32_t* seed_offsets,
                            const int32_t* seed_index, const double* seed_time, int mode, double tol, int max_rounds,
                            void* out, int out_type, ts_eik_stats* stats) {
    const int precision = precision_of<Real>();
    std::vector<std::unique_ptr<host::Grid>> g(n_grids);
    std::vector<std::unique_ptr<host::Metric>> m(n_grids);
    EngineJob job;
    std::vector<Real*> slow_d(n_grids, nullptr);
    size_t total = 0;
    for (int q = 0; q < n_grids; q++) {
        if (const char* bad = host::Grid::validate(grids[q])) return ctx->fail(TS_E_ARG, std::string("grid ") + std::to_string(q) + ": " + bad);
        g[q].reset(new host::Grid(grids[q]));
        m[q].reset(new host::Metric(*g[q]));
        job.grids.push_back(g[q].get());
        job.metrics.push_back(m[q].get());
        total += size_t(g[q]->count());
    }
    // Slowness of every grid in one device buffer, in the solve's precision.
    Real* sl = static_cast<Real*>(ctx->buf("multi.slowness", sizeof(Real) * total));
    if (!sl) return TS_E_NOMEM;
    {
        std::vector<Real> tmp(total);
        size_t o = 0;
        for (int q = 0; q < n_grids; q++) {
            slow_d[q] = sl + o;
            for (int64_t e = 0; e < g[q]->count(); e++) tmp[o + e] = Real(slowness[q][e]);
            o += size_t(g[q]->count());
        }
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(sl, tmp.data(), sizeof(Real) * total, cudaMemcpyHostToDevice, ctx->stream));
        TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    job.tol = tol;
    job.wake_rel = mode == TS_MODE_FAST ? TS_WAKE_REL : 0.0;
    job.tile = precision == TS_PRECISION_F64 ? ctx->tile_f64 : ctx->tile_f32;
    int64_t out_total = 0;
    for (int f = 0; f < n_fields; f++) {
        int gi = field_grid[f];
        if (gi < 0 || gi >= n_grids) return ctx->fail(TS_E_ARG, "field_grid out of range");
        EngineField ef;
        ef.grid = gi;
        ef.slowness = slow_d[gi];
        const host::Grid& gg = *g[gi];
        std::map<int32_t, double> merged;
        for (int q = seed_offsets[f]; q < seed_offsets[f + 1]; q++) {
            if (uint32_t(seed_index[q]) >= uint64_t(gg.count())) continue;
            auto it = merged.find(seed_index[q]);
            if (it == merged.end() || seed_time[q] < it->second) merged[seed_index[q]] = seed_time[q];
        }
        if (merged.empty()) return ctx->fail(TS_E_NOSEEDS, "no seed nodes for field " + std::to_string(f));
        for (auto& kv : merged) {
            ef.seed_idx.push_back(kv.first);
            ef.seed_t.push_back(kv.second);
        }
        ef.cap = max_rounds > 0 ? max_rounds : std::max(32, (gg.nx + gg.ny + gg.nz) / 4);
        job.fields.push_back(std::move(ef));
        out_total += gg.count();
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    int rc = engine_run<Real>(ctx, job, stats);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int r0 = 0, r1 = 0;
    for (auto& ef : job.fields) {
        r0 = std::max(r0, ef.rounds[0]);
        r1 = std::max(r1, ef.rounds[1]);
    }
    if (stats) {
        stats->device_ms = ms;
        stats->rounds[0] = r0;
        stats->rounds[1] = r1;
    }
    ctx->stats = std::to_string(r0) + "+" + std::to_string(r1) + " rounds of 8 sweeps";
    if (rc) return rc;
    for (auto& ef : job.fields)
        if (ef.status != 1) return ctx->fail(TS_E_UNSETTLED, "sweeping not settled within the round cap");
    if (out_type == TS_OUT_NONE) return TS_OK;
    return fields_to_dense_host(ctx, job, precision, out, out_type);
}

}  // namespace eik
}  // namespace ts

extern "C" {

int ts_eik_solve_multi(ts_ctx* ctx, int32_t n_grids, const ts_grid* grids, const double* const* slowness,
                       int32_t n_fields, const int32_t* field_grid, const int32_t* seed_offsets, const int32_t* seed_index,
                       const double* seed_time, int32_t precision, int32_t mode, double tol, int32_t max_rounds,
                       void* out, int32_t out_type, ts_eik_stats* stats) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    ts_eik_stats local{};
    if (!stats) stats = &local;
    *stats = ts_eik_stats{};
    if (n_grids <= 0 || !grids || !slowness || n_fields <= 0 || !field_grid || !seed_offsets)
        return ctx->fail(TS_E_ARG, "null array or empty batch");
    if (seed_offsets[n_fields] > 0 && (!seed_index || !seed_time)) return ctx->fail(TS_E_ARG, "null seed arrays");
    if (mode != TS_MODE_ENGINE && mode != TS_MODE_FAST) return ctx->fail(TS_E_ARG, "mode must be engine or fast");
    if (out_type != TS_OUT_F64 && out_type != TS_OUT_F32 && out_type != TS_OUT_NONE)
        return ctx->fail(TS_E_ARG, "unknown output type");
    if (out_type != TS_OUT_NONE && !out) return ctx->fail(TS_E_ARG, "null output");
    if (!(tol >= 0)) return ctx->fail(TS_E_ARG, "tolerance must be >= 0");
    if (precision == TS_PRECISION_F64)
        return ts::eik::solve_multi_impl<double>(ctx, n_grids, grids, slowness, n_fields, field_grid, seed_offsets,
                                                 seed_index, seed_time, mode, tol, max_rounds, out, out_type, stats);
    if (precision == TS_PRECISION_F32)
        return ts::eik::solve_multi_impl<ts::Pair>(ctx, n_grids, grids, slowness, n_fields, field_grid, seed_offsets,
                                                seed_index, seed_time, mode, tol, max_rounds, out, out_type, stats);
    return ctx->fail(TS_E_ARG, "precision must be 64 or 32");
}

int ts_engine_set_graph(ts_ctx* ctx, int32_t enable) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    ctx->use_graph = enable != 0;
    if (!ctx->use_graph) ctx->drop_graph();
    return TS_OK;
}

int32_t ts_engine_graph_replays(ts_ctx* ctx) { return ctx ? ctx->graph_replays : 0; }

int ts_engine_autotune(ts_ctx* ctx, int32_t n_grids, const ts_grid* grids, const double* const* slowness,
                       int32_t n_fields, const int32_t* field_grid, const int32_t* seed_offsets, const int32_t* seed_index,
                       const double* seed_time, int32_t precision, int32_t mode, int32_t repeats, int32_t* best_tile,
                       int32_t* best_scheduler, double* ms_per_shape, int32_t cap) {
    if (!ctx || !best_tile) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    const auto& shapes = ts::eik::tile_shapes();
    int best = -1, best_sched = 0;
    double best_ms = INFINITY;
    const int keep64 = ctx->tile_f64, keep32 = ctx->tile_f32, keep_sched = ctx->scheduler;
    const bool keep_graph = ctx->use_graph;
    ctx->use_graph = false;
    auto restore = [&]() {
        ctx->tile_f64 = keep64;
        ctx->tile_f32 = keep32;
        ctx->scheduler = keep_sched;
        ctx->use_graph = keep_graph;
    };
    // Every (shape, scheduler) pair; entry 2·q + scheduler of ms_per_shape.
    for (size_t q = 0; q < shapes.size(); q++) {
        for (int sched = 0; sched < 2; sched++) {
            if (precision == TS_PRECISION_F64) ctx->tile_f64 = shapes[q].id;
            else ctx->tile_f32 = shapes[q].id;
            ctx->scheduler = sched;
            double ms = INFINITY;
            for (int r = 0; r < std::max(1, repeats); r++) {
                ts_eik_stats st{};
                int rc = ts_eik_solve_multi(ctx, n_grids, grids, slowness, n_fields, field_grid, seed_offsets,
                                            seed_index, seed_time, precision, mode, 1e-7, 0, nullptr, TS_OUT_NONE, &st);
                if (rc) {
                    restore();
                    return rc;
                }
                ms = std::min(ms, st.device_ms);
            }
            const int32_t slot = int32_t(2 * q + sched);
            if (ms_per_shape && slot < cap) ms_per_shape[slot] = ms;
            if (ms < best_ms) {
                best_ms = ms;
                best = shapes[q].id;
                best_sched = sched;
            }
        }
    }
    restore();
    if (precision == TS_PRECISION_F64) ctx->tile_f64 = best;
    else ctx->tile_f32 = best;
    ctx->scheduler = best_sched;
    ctx->drop_graph();
    *best_tile = best;
    if (best_scheduler) *best_scheduler = best_sched;
    return TS_OK;
}

}  // extern "C"
