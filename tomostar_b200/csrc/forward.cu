// ts_forward: RayKernels.Compute for travel times (Tomography/RayKernels.cs:30-115) with every
// table solved and kept on the device. The tables of the (station, phase) pairs the arrivals use
// are solved by the engine in one launch (TravelTimeTableSet.Build, Forward/TravelTimeTable.cs:264-308,
// seeds by PointSource at the station, :335/:373), rounded to float32 as TravelTimeTable.Write does
// (:73), and every arrival is traced on its table (RayKernels.cs:67-107).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <map>
#include <vector>

#include "ctx.h"
#include "eik_engine.h"
#include "host_geo.h"
#include "rays.h"

namespace ts {
namespace fwd {

template <typename Real>
static int upload_slowness(ts_ctx* ctx, const double* src, size_t count, Real* dst) {
    std::vector<Real> tmp(count);
    for (size_t q = 0; q < count; q++) tmp[q] = Real(src[q]);
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(dst, tmp.data(), count * sizeof(Real), cudaMemcpyHostToDevice, ctx->stream));
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return TS_OK;
}

// The float32 tables of `tables` ((phase, source) pairs; sources hold lon, lat, depth) on g, solved
// by the engine in batches that fit the device next to the tables, each rounded to float32 into its
// slot of `tab` (n_nodes floats per table): TravelTimeTableSet.Build (Forward/TravelTimeTable.cs:264-308)
// with the seeds of PointSource at the source (:373). mode: TS_MODE_ENGINE (the reference's fields to
// the bit) or TS_MODE_FAST (within 1e-10 relative of them, about half the node evaluations).
template <typename Real>
int solve_tables(ts_ctx* ctx, const host::Grid& g, const double* slowness, int n_phases, int mode,
                 const std::vector<std::pair<int, int>>& tables, const double* sources, float* tab,
                 ts_eik_stats* stats) {
    host::Metric m(g);
    const int64_t n = g.count();
    const int nt = int(tables.size());
    // Slowness per phase on the device.
    Real* slow_d = static_cast<Real*>(ctx->buf("fwd.slowness", sizeof(Real) * size_t(n) * n_phases));
    if (!slow_d) return TS_E_NOMEM;
    int rc = upload_slowness<Real>(ctx, slowness, size_t(n) * n_phases, slow_d);
    if (rc) return rc;
    // Seeds: PointSource at each source (TravelTimeTable.cs:373).
    std::vector<std::vector<int32_t>> sidx(nt);
    std::vector<std::vector<double>> st(nt);
    for (int t = 0; t < nt; t++) {
        const double* sp = sources + 3 * tables[t].second;
        const double* sl = slowness + size_t(n) * tables[t].first;
        std::vector<int32_t> idx(8192);
        std::vector<double> tv(8192);
        int c = host::point_source(g, sl, sp[0], sp[1], sp[2], 0, 3, idx.data(), tv.data(), 8192);
        if (c > 8192) {
            idx.resize(c);
            tv.resize(c);
            c = host::point_source(g, sl, sp[0], sp[1], sp[2], 0, 3, idx.data(), tv.data(), c);
        }
        // TrySolve's merge (EikonalOpenCl.cs:150-163): PointSource gives distinct nodes in order.
        sidx[t].assign(idx.begin(), idx.begin() + c);
        st[t].assign(tv.begin(), tv.begin() + c);
        if (c == 0) return ctx->fail(TS_E_NOSEEDS, "no seed nodes for source " + std::to_string(tables[t].second));
    }
    const int precision = precision_of<Real>();
    const int tile = is_f64<Real>() ? ctx->tile_f64 : ctx->tile_f32;
    const size_t per_field = size_t(eik::field_layout(g, tile, precision).bytes(precision));
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    cudaGetLastError();
    free_b += ctx->bufs.count("eng.fields") ? ctx->bufs["eng.fields"].n : 0;  // reused by the batches
    const size_t room = free_b > (size_t(4) << 30) ? free_b - (size_t(4) << 30) : free_b / 2;
    const int batch = int(std::max<size_t>(1, std::min<size_t>(size_t(std::max(1, nt)), room / per_field)));
    const int cap = std::max(32, (g.nx + g.ny + g.nz) / 4);
    int r0 = 0, r1 = 0;
    double field_ms = 0;
    for (int t0 = 0; t0 < nt; t0 += batch) {
        const int t1 = std::min(nt, t0 + batch);
        eik::EngineJob job;
        job.grids.push_back(&g);
        job.metrics.push_back(&m);
        job.tol = 1e-7;  // SphericalEikonal.SettleTolerance
        job.wake_rel = mode == TS_MODE_FAST ? TS_WAKE_REL : 0.0;
        job.tile = tile;
        for (int t = t0; t < t1; t++) {
            eik::EngineField ef;
            ef.grid = 0;
            ef.slowness = slow_d + size_t(n) * tables[t].first;
            ef.seed_idx = sidx[t];
            ef.seed_t = st[t];
            ef.cap = cap;
            job.fields.push_back(ef);
        }
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, ctx->stream);
        ts_eik_stats bst{};
        rc = eik::engine_run<Real>(ctx, job, &bst);
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        field_ms += ms;
        if (stats) {
            stats->node_updates += bst.node_updates;
            stats->tile_visits += bst.tile_visits;
            stats->launches += bst.launches;
            stats->kernel_ms += bst.kernel_ms;
        }
        if (rc) return rc;
        for (auto& ef : job.fields) {
            if (ef.status != 1)
                return ctx->fail(TS_E_UNSETTLED, "sweeping not settled after " + std::to_string(cap) + " rounds");
            r0 = std::max(r0, ef.rounds[0]);
            r1 = std::max(r1, ef.rounds[1]);
        }
        rc = eik::fields_to_dense_f32_device(ctx, job, precision, tab + size_t(t0) * n);
        if (rc) return rc;
    }
    if (stats) {
        stats->rounds[0] = r0;
        stats->rounds[1] = r1;
        stats->device_ms = field_ms;
    }
    ctx->stats = std::to_string(r0) + "+" + std::to_string(r1) + " rounds of 8 sweeps";
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->release("eng.fields");
    return TS_OK;
}

template int solve_tables<double>(ts_ctx*, const host::Grid&, const double*, int, int, const std::vector<std::pair<int, int>>&,
                                  const double*, float*, ts_eik_stats*);
template int solve_tables<Pair>(ts_ctx*, const host::Grid&, const double*, int, int, const std::vector<std::pair<int, int>>&,
                                 const double*, float*, ts_eik_stats*);

template <typename Real>
static int forward_impl(ts_ctx* ctx, const ts_grid* fwd_def, const double* slowness, int n_phases, int mode,
                        const ts_grid* inv_def, int n_stations, const double* stations, int n_events,
                        const double* events, int n_arr, const int32_t* arr_event, const int32_t* arr_station,
                        const int32_t* arr_phase, double step_km, ts_rows** out, ts_eik_stats* stats) {
    host::Grid g(*fwd_def), gi(*inv_def);
    const int64_t n = g.count();
    const auto t_begin = std::chrono::steady_clock::now();
    // Tables of the (station, phase) pairs in use, ordered by phase then station (TravelTimeTable.cs:319):
    // table_id[phase * n_stations + station], -1 where unused.
    std::vector<int> table_id(size_t(n_phases) * std::max(1, n_stations), -1);
    for (int a = 0; a < n_arr; a++) {
        if (arr_event[a] < 0 || arr_event[a] >= n_events || arr_station[a] < 0 || arr_station[a] >= n_stations ||
            arr_phase[a] < 0 || arr_phase[a] >= n_phases)
            return ctx->fail(TS_E_ARG, "arrival " + std::to_string(a) + " refers outside the inputs");
        table_id[size_t(arr_phase[a]) * n_stations + arr_station[a]] = 0;
    }
    std::vector<std::pair<int, int>> tables;
    for (int ph = 0; ph < n_phases; ph++)
        for (int st = 0; st < n_stations; st++) {
            int& id = table_id[size_t(ph) * n_stations + st];
            if (id < 0) continue;
            id = int(tables.size());
            tables.push_back({ph, st});
        }
    const int nt = int(tables.size());
    std::vector<double> table_station(3 * std::max(1, nt));
    for (int t = 0; t < nt; t++)
        for (int c = 0; c < 3; c++) table_station[3 * t + c] = stations[3 * tables[t].second + c];
    float* tab = nullptr;
    if (nt > 0) {
        tab = static_cast<float*>(ctx->buf("fwd.tables", sizeof(float) * size_t(n) * nt));
        if (!tab) return TS_E_NOMEM;
    }
    int rc = solve_tables<Real>(ctx, g, slowness, n_phases, mode, tables, stations, tab, stats);
    if (rc) return rc;
    const std::string table_stats = ctx->stats;
    const auto t_tables = std::chrono::steady_clock::now();
    // Arrivals → rays (the engine's field buffers were released for the rows).
    std::vector<int32_t> table_of(std::max(1, n_arr));
    std::vector<double> ev(3 * std::max(1, n_arr));
    for (int a = 0; a < n_arr; a++) {
        table_of[a] = table_id[size_t(arr_phase[a]) * n_stations + arr_station[a]];
        for (int c = 0; c < 3; c++) ev[3 * a + c] = events[3 * arr_event[a] + c];
    }
    if (!(step_km > 0)) step_km = 0.5 * std::min(g.min_spacing_km(), gi.min_spacing_km());  // RayKernels.cs:62
    std::vector<int32_t> table_phase(std::max(1, nt));
    for (int t = 0; t < nt; t++) table_phase[t] = tables[t].first;
    rays::RayStats rs;
    rc = rays::trace_on_device(ctx, g, tab, std::max(1, nt), table_station.data(), gi, n_arr, table_of.data(),
                               ev.data(), step_km, out, &rs, table_phase.data());
    if (rc) return rc;
    // The step's timing in the context's stats text (ts_last_stats): the tables' call, then the rays'.
    using ms = std::chrono::duration<double, std::milli>;
    const auto t_end = std::chrono::steady_clock::now();
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "; tables %.1f ms; rays %.1f ms (host set-up %.1f ms, ray pipeline %.1f ms, on the device %.1f ms, "
                  "%d chunks, %llu steps)",
                  ms(t_tables - t_begin).count(), ms(t_end - t_tables).count(), rs.setup_ms, rs.wall_ms, rs.device_ms,
                  rs.chunks, rs.steps);
    ctx->stats = table_stats + buf;
    return TS_OK;
}

}  // namespace fwd
}  // namespace ts

extern "C" int ts_forward(ts_ctx* ctx, const ts_grid* fwd, const double* slowness, int32_t n_phases,
                          const ts_grid* inv, int32_t n_stations, const double* stations, int32_t n_events,
                          const double* events, int32_t n_arrivals, const int32_t* arr_event,
                          const int32_t* arr_station, const int32_t* arr_phase, int32_t precision, int32_t mode,
                          double step_km, ts_rows** out, ts_eik_stats* stats) {
    if (!ctx || !out) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = nullptr;
    if (stats) *stats = ts_eik_stats{};
    if (!fwd || !inv) return ctx->fail(TS_E_ARG, "grid is null");
    if (const char* bad = ts::host::Grid::validate(*fwd)) return ctx->fail(TS_E_ARG, bad);
    if (const char* bad = ts::host::Grid::validate(*inv)) return ctx->fail(TS_E_ARG, bad);
    if (fwd->depth_km || inv->depth_km) return ctx->fail(TS_E_ARG, "the forward step needs uniform grids");
    if (!slowness || n_phases <= 0 || n_stations < 0 || n_events < 0 || n_arrivals < 0)
        return ctx->fail(TS_E_ARG, "bad sizes");
    if (n_arrivals > 0 && (!stations || !events || !arr_event || !arr_station || !arr_phase))
        return ctx->fail(TS_E_ARG, "null arrival arrays");
    if (mode != TS_MODE_ENGINE && mode != TS_MODE_FAST) return ctx->fail(TS_E_ARG, "mode must be engine or fast");
    if (precision == TS_PRECISION_F64)
        return ts::fwd::forward_impl<double>(ctx, fwd, slowness, n_phases, mode, inv, n_stations, stations, n_events, events,
                                             n_arrivals, arr_event, arr_station, arr_phase, step_km, out, stats);
    if (precision == TS_PRECISION_F32)
        return ts::fwd::forward_impl<ts::Pair>(ctx, fwd, slowness, n_phases, mode, inv, n_stations, stations, n_events, events,
                                            n_arrivals, arr_event, arr_station, arr_phase, step_km, out, stats);
    return ctx->fail(TS_E_ARG, "precision must be 64 or 32");
}
