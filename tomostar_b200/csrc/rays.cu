// Rays and Jacobian rows on the device: RayTracing.Backtrack (Forward/RayTracing.cs:73-111),
// RayTracing.Kernel (:118-159) and RayKernels' row finalisation (Tomography/RayKernels.cs:79-97).
//
// Rays are taken in order of their table (so that a table's float32 nodes stay in L2 while its rays
// are traced) in chunks sized by a record budget; each ray's record room is its own estimate.
// Kernels, none with atomics:
//   trace_kernel  one thread per ray: steepest descent on the station's float32 table, each new
//                 polyline segment integrated at once against the trilinear basis of the inversion
//                 grid. Pieces falling in the same inversion cell are summed before a record
//                 (node, length) is written, and a node shared with the next cell (a face
//                 neighbour) keeps its running sum, so a ray writes about one record per node.
//                 A step's gradient loads its six evaluations' 48 corners together (one memory
//                 latency instead of six dependent ones).
//   merge_kernel  one warp per ray: sorts the ray's records by node (bitonic, shared memory, the
//                 record index breaking ties so equal nodes keep visit order), sums each node's
//                 lengths in that order and writes the unique nodes ascending, lengths as float32.
//   stage_kernel  one warp per ray: appends the chunk's rows to a staging area (chunk order).
//   emit_kernel   one warp per ray: copies every row from the staging area into the CSR arrays at
//                 its offset in arrival order, once all chunks are traced.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "ctx.h"
#include "geo_dev.cuh"
#include "host_geo.h"
#include "rays.h"

namespace ts {
namespace rays {

using geo::GeoPt;
using geo::RGrid;
using geo::V3;

constexpr int kDropped = -1;   // the reference returns null: the row is left out
constexpr int kOverflow = -2;  // more records than the chunk's capacity: traced again with more

struct TraceArgs {
    RGrid fwd, inv;
    const float* tables;
    int64_t table_n;
    const float* const* table_ptr;  // when set: table t at table_ptr[t] (tables in separate buffers)
    const double* table_station;  // 3 per table
    const int* table_of;          // per ray
    const double* events;         // 3 per ray
    const int* ray_of;            // global ray index of each chunk slot
    int nrays;                    // chunk slots
    double step_km, piece_km;
    const int64_t* rec_base;      // per chunk slot: first record of its room
    const int* rec_cap;           // per chunk slot: records it may write
    int* rec_node;                // the chunk's records
    double* rec_val;
    int* rec_count;               // per chunk slot
    double* tcg;                  // 4 per ray (global index)
    double* outside;              // per ray (global index): time outside the inversion grid
    unsigned long long* steps;    // back-tracing steps of every ray traced (the gathers' unit)
    int bg_n;                     // > 0: the extended domain's background (depths, Vp, Vs at bg)
    const double* bg;
    const int* table_phase;       // per table: 0 P (Vp), 1 S (Vs)
};

// Per-ray record writer with the current inversion cell's eight accumulators.
struct Recorder {
    int ci = -1, cj = 0, ck = 0;
    unsigned touched = 0;
    double acc[8];
    int count = 0;
    bool overflow = false;
    double outside = 0;           // RayRow.OutsideTime
    const double* bgv = nullptr;  // the background's velocity of the ray's phase

    // The record (node, running sum) of corner n of the current cell.
    TS_DEVINL void record(const TraceArgs& a, int r, int n) {
        if (count >= a.rec_cap[r]) {
            overflow = true;
            return;
        }
        const int di = n & 1, dj = (n >> 1) & 1, dk = n >> 2;
        const int64_t slot = a.rec_base[r] + count;
        a.rec_node[slot] = int((ck + dk) * (int64_t(a.inv.nx) * a.inv.ny) + int64_t(cj + dj) * a.inv.nx + (ci + di));
        a.rec_val[slot] = acc[n];
        count++;
    }

    TS_DEVINL void flush(const TraceArgs& a, int r) {
        if (ci < 0 || !touched) return;
#pragma unroll
        for (int n = 0; n < 8; n++)
            if ((touched >> n) & 1u) record(a, r, n);
        touched = 0;
    }

    // Moving into the face neighbour along axis bit B (UP: to the larger index), the four corners the
    // two cells share keep their running sums, so a node's pieces add up in visit order with no record
    // in between; the other four are written.
    template <int B, bool UP>
    TS_DEVINL void carry(const TraceArgs& a, int r) {
        double nacc[8];
        unsigned nt = 0;
#pragma unroll
        for (int n = 0; n < 8; n++) nacc[n] = 0.0;
#pragma unroll
        for (int n = 0; n < 8; n++) {
            if (!((touched >> n) & 1u)) continue;
            if (UP ? (n & B) != 0 : (n & B) == 0) {
                nacc[n ^ B] = acc[n];
                nt |= 1u << (n ^ B);
            } else {
                record(a, r, n);
            }
        }
#pragma unroll
        for (int n = 0; n < 8; n++) acc[n] = nacc[n];
        touched = nt;
    }

    // RayTracing.Kernel for one polyline segment (RayTracing.cs:133-157), from its end points in
    // Cartesian form (the back-tracing loop has converted both already: the same values).
    TS_DEVINL void segment(const TraceArgs& a, int r, V3 A, V3 B) {
        V3 d = geo::sub(B, A);
        double len = geo::norm(d);
        if (len <= 0) return;
        int pieces = max(1, int(ceil(len / a.piece_km)));
        double dl = len / pieces;
        for (int q = 0; q < pieces; q++) {
            GeoPt mid = geo::from_cartesian(geo::add(A, geo::scale(d, (q + 0.5) / pieces)));
            // The extended domain (RayTracing.cs:141-145): a piece outside the inversion grid is
            // not attributed; its length times the background's slowness is time outside.
            if (a.bg_n > 0 && !geo::contains(a.inv, mid.lon, mid.lat, mid.dep, 1e-6)) {
                outside += dl * (1 / geo::background_1d(a.bg, bgv, a.bg_n, mid.dep));
                continue;
            }
            double fx, fy, fz;
            geo::fractional(a.inv, mid.lon, mid.lat, mid.dep, fx, fy, fz);
            int i0, j0, k0;
            double w[8];
            geo::weights(a.inv, fx, fy, fz, i0, j0, k0, w);
            if (i0 != ci || j0 != cj || k0 != ck) {
                const int di = i0 - ci, dj = j0 - cj, dk = k0 - ck;
                if (ci >= 0 && abs(di) + abs(dj) + abs(dk) == 1) {
                    if (di == 1) carry<1, true>(a, r);
                    else if (di == -1) carry<1, false>(a, r);
                    else if (dj == 1) carry<2, true>(a, r);
                    else if (dj == -1) carry<2, false>(a, r);
                    else if (dk == 1) carry<4, true>(a, r);
                    else carry<4, false>(a, r);
                } else {
                    flush(a, r);
#pragma unroll
                    for (int n = 0; n < 8; n++) acc[n] = 0.0;
                }
                ci = i0; cj = j0; ck = k0;
            }
#pragma unroll
            for (int n = 0; n < 8; n++) {
                if (w[n] == 0) continue;
                acc[n] += dl * w[n] * 1.0;
                touched |= 1u << n;
            }
        }
    }
};

__global__ void __launch_bounds__(128) trace_kernel(TraceArgs a) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrays) return;
    const int ray = a.ray_of[r];
    const int tab = a.table_of[ray];
    const float* tb = a.table_ptr ? a.table_ptr[tab] : a.tables + int64_t(tab) * a.table_n;
    const RGrid& g = a.fwd;
    const double st_lon = a.table_station[3 * tab], st_lat = a.table_station[3 * tab + 1];
    const double st_dep = fmin(fmax(a.table_station[3 * tab + 2], g.min_dep), g.dep_last);
    const GeoPt ev{a.events[3 * ray], a.events[3 * ray + 1], a.events[3 * ray + 2]};
    double* tcg = a.tcg + 4 * int64_t(ray);
    a.outside[ray] = 0;

    // Backtrack (RayTracing.cs:75-110).
    V3 station = geo::to_cartesian(st_lon, st_lat, st_dep);
    V3 p = geo::to_cartesian(ev.lon, ev.lat, ev.dep);
    double t0 = geo::table_time_b(g, tb, ev.lon, ev.lat, ev.dep);
    tcg[0] = t0;
    if (!isfinite(t0)) {
        a.rec_count[r] = kDropped;
        return;
    }
    geo::table_gradient_b(g, tb, ev.lon, ev.lat, ev.dep, tcg[1], tcg[2], tcg[3]);
    const double step = a.step_km;
    const int max_steps = 20 * int(ceil(geo::norm(geo::sub(p, station)) / step + 10));
    double last_t = t0;
    int stalls = 0;
    Recorder rec;
    if (a.bg_n > 0) rec.bgv = a.bg + (a.table_phase[tab] == 0 ? 1 : 2) * a.bg_n;
    // The steps this ray takes, added to the launch's count on every way out.
    struct StepCount {
        unsigned long long* total;
        unsigned long long n = 0;
        TS_DEVINL ~StepCount() { atomicAdd(total, n); }
    } taken{a.steps};
    V3 prev = p;  // the polyline's last point (Cartesian of the event, then of each step's point)
    for (int s = 0; s < max_steps; s++) {
        if (geo::norm(geo::sub(p, station)) <= 1.5 * step) break;
        taken.n++;
        GeoPt gp = geo::from_cartesian(p);
        double ge, gn, gz;
        geo::table_gradient_b(g, tb, gp.lon, gp.lat, gp.dep, ge, gn, gz);
        if (!isfinite(ge) || !isfinite(gn) || !isfinite(gz)) {
            a.rec_count[r] = kDropped;
            return;
        }
        // LocalFrame (GeoMath.cs:71-80) and the step against the gradient.
        double sl, cl, so, co;
        sincos(gp.lat * kDeg2Rad, &sl, &cl);
        sincos(gp.lon * kDeg2Rad, &so, &co);
        V3 e{-so, co, 0}, nn{-sl * co, -sl * so, cl}, up{cl * co, cl * so, sl};
        V3 grad = geo::add(geo::add(geo::scale(e, ge), geo::scale(nn, gn)), geo::scale(up, -gz));
        double nrm = geo::norm(grad);
        if (nrm < 1e-12) {
            a.rec_count[r] = kDropped;
            return;
        }
        p = geo::sub(p, geo::scale(grad, step / nrm));
        GeoPt q = geo::from_cartesian(p);
        q.lon = fmin(fmax(geo::unwrap_lon(q.lon, g.centre_lon), g.min_lon), g.lon_last);
        q.lat = fmin(fmax(q.lat, g.min_lat), g.lat_last);
        q.dep = fmin(fmax(q.dep, g.min_dep), g.dep_last);
        p = geo::to_cartesian(q.lon, q.lat, q.dep);
        rec.segment(a, r, prev, p);
        prev = p;
        double t = geo::table_time_b(g, tb, q.lon, q.lat, q.dep);
        if (!(t < last_t)) {
            if (++stalls > 20) {
                a.rec_count[r] = kDropped;
                return;
            }
        } else {
            stalls = 0;
        }
        last_t = fmin(last_t, t);
    }
    rec.segment(a, r, prev, station);
    rec.flush(a, r);
    a.outside[ray] = rec.outside;
    a.rec_count[r] = rec.overflow ? kOverflow : rec.count;
}

// Backtrack + Kernel with one warp per ray, for calls too small to fill the device with a thread per
// ray (a serving completion traces a few hundred): the lanes share each step's corner loads and sum
// the six gradient evaluations side by side (table_gradient_w), every lane carries the ray's state
// through the same arithmetic, and lane 0 integrates the segments and writes the records. The values
// are those of trace_kernel, so the rows are the same bits.
__global__ void __launch_bounds__(128) trace_warp_kernel(TraceArgs a) {
    const int lane = threadIdx.x & 31;
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= a.nrays) return;  // the whole warp
    const bool lead = lane == 0;
    const int ray = a.ray_of[r];
    const int tab = a.table_of[ray];
    const float* tb = a.table_ptr ? a.table_ptr[tab] : a.tables + int64_t(tab) * a.table_n;
    const RGrid& g = a.fwd;
    const double st_lon = a.table_station[3 * tab], st_lat = a.table_station[3 * tab + 1];
    const double st_dep = fmin(fmax(a.table_station[3 * tab + 2], g.min_dep), g.dep_last);
    const GeoPt ev{a.events[3 * ray], a.events[3 * ray + 1], a.events[3 * ray + 2]};
    double* tcg = a.tcg + 4 * int64_t(ray);
    if (lead) a.outside[ray] = 0;

    V3 station = geo::to_cartesian(st_lon, st_lat, st_dep);
    V3 p = geo::to_cartesian(ev.lon, ev.lat, ev.dep);
    double t0 = geo::table_time_w(g, tb, ev.lon, ev.lat, ev.dep, lane);
    if (lead) tcg[0] = t0;
    if (!isfinite(t0)) {
        if (lead) a.rec_count[r] = kDropped;
        return;
    }
    double g0e, g0n, g0z;
    geo::table_gradient_w(g, tb, ev.lon, ev.lat, ev.dep, g0e, g0n, g0z, lane);
    if (lead) {
        tcg[1] = g0e;
        tcg[2] = g0n;
        tcg[3] = g0z;
    }
    const double step = a.step_km;
    const int max_steps = 20 * int(ceil(geo::norm(geo::sub(p, station)) / step + 10));
    double last_t = t0;
    int stalls = 0;
    Recorder rec;
    if (a.bg_n > 0) rec.bgv = a.bg + (a.table_phase[tab] == 0 ? 1 : 2) * a.bg_n;
    unsigned long long taken = 0;
    V3 prev = p;
    bool dropped = false;
    for (int s = 0; s < max_steps; s++) {
        if (geo::norm(geo::sub(p, station)) <= 1.5 * step) break;
        taken++;
        GeoPt gp = geo::from_cartesian(p);
        double ge, gn, gz;
        geo::table_gradient_w(g, tb, gp.lon, gp.lat, gp.dep, ge, gn, gz, lane);
        if (!isfinite(ge) || !isfinite(gn) || !isfinite(gz)) {
            dropped = true;
            break;
        }
        double sl, cl, so, co;
        sincos(gp.lat * kDeg2Rad, &sl, &cl);
        sincos(gp.lon * kDeg2Rad, &so, &co);
        V3 e{-so, co, 0}, nn{-sl * co, -sl * so, cl}, up{cl * co, cl * so, sl};
        V3 grad = geo::add(geo::add(geo::scale(e, ge), geo::scale(nn, gn)), geo::scale(up, -gz));
        double nrm = geo::norm(grad);
        if (nrm < 1e-12) {
            dropped = true;
            break;
        }
        p = geo::sub(p, geo::scale(grad, step / nrm));
        GeoPt q = geo::from_cartesian(p);
        q.lon = fmin(fmax(geo::unwrap_lon(q.lon, g.centre_lon), g.min_lon), g.lon_last);
        q.lat = fmin(fmax(q.lat, g.min_lat), g.lat_last);
        q.dep = fmin(fmax(q.dep, g.min_dep), g.dep_last);
        p = geo::to_cartesian(q.lon, q.lat, q.dep);
        if (lead) rec.segment(a, r, prev, p);
        prev = p;
        double t = geo::table_time_w(g, tb, q.lon, q.lat, q.dep, lane);
        if (!(t < last_t)) {
            if (++stalls > 20) {
                dropped = true;
                break;
            }
        } else {
            stalls = 0;
        }
        last_t = fmin(last_t, t);
    }
    if (!lead) return;
    atomicAdd(a.steps, taken);
    if (dropped) {
        a.rec_count[r] = kDropped;
        return;
    }
    rec.segment(a, r, prev, station);
    rec.flush(a, r);
    a.outside[ray] = rec.outside;
    a.rec_count[r] = rec.overflow ? kOverflow : rec.count;
}

// One warp per ray: sort records by (node, record index), sum each node in record order, write
// the unique nodes ascending. P is the power-of-two sort size of one warp's shared memory.
// A pass handles the rays with lo < records <= P; the first pass (lo = 0) also writes the empty
// and dropped rows and marks the rays left for a larger pass.
__global__ void merge_kernel(const int* __restrict__ rec_node, const double* __restrict__ rec_val,
                             const int* __restrict__ rec_count, const int64_t* __restrict__ rec_base, int nrays,
                             int P, int lo, int* __restrict__ out_node, float* __restrict__ out_len,
                             int* __restrict__ nnz) {
    extern __shared__ unsigned long long keys_all[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    unsigned long long* keys = keys_all + size_t(warp) * P;
    for (int r = blockIdx.x * wpb + warp; r < nrays; r += gridDim.x * wpb) {
        int c = rec_count[r];
        if (c <= lo) {
            if (lane == 0 && lo == 0) nnz[r] = c;  // 0, kDropped or kOverflow
            continue;
        }
        if (c > P) {
            if (lane == 0 && lo == 0) nnz[r] = kOverflow;  // for the larger pass to overwrite
            continue;
        }
        int n2 = 32;
        while (n2 < c) n2 <<= 1;
        const int64_t base = rec_base[r];
        for (int q = lane; q < n2; q += 32)
            keys[q] = q < c ? (static_cast<unsigned long long>(unsigned(rec_node[base + q])) << 32) | unsigned(q)
                            : ~0ull;
        __syncwarp();
        for (int k = 2; k <= n2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int q = lane; q < n2; q += 32) {
                    int l = q ^ j;
                    if (l > q) {
                        unsigned long long x = keys[q], y = keys[l];
                        bool up = (q & k) == 0;
                        if ((x > y) == up) {
                            keys[q] = y;
                            keys[l] = x;
                        }
                    }
                }
                __syncwarp();
            }
        }
        // Segment starts, ranked by a running warp scan; each start sums its node in record order.
        int written = 0;
        for (int q0 = 0; q0 < c; q0 += 32) {
            int q = q0 + lane;
            bool start = false;
            unsigned node = 0;
            if (q < c) {
                node = unsigned(keys[q] >> 32);
                start = q == 0 || unsigned(keys[q - 1] >> 32) != node;
            }
            unsigned m = __ballot_sync(0xffffffffu, start);
            if (start) {
                int rank = written + __popc(m & ((1u << lane) - 1u));
                double sum = 0;
                for (int e = q; e < c && unsigned(keys[e] >> 32) == node; e++) sum += rec_val[base + unsigned(keys[e])];
                out_node[base + rank] = int(node);
                out_len[base + rank] = float(sum);  // RayKernels.cs:97: (float)kernel[x]
            }
            written += __popc(m);
        }
        if (lane == 0) nnz[r] = written;
        __syncwarp();
    }
}

// Exclusive scan of the chunk's row sizes (negative = empty row) in one block; total and the
// number of rows still marked for the large pass go to sums[0], sums[1].
__global__ void scan_kernel(const int* __restrict__ nnz, int n, int* __restrict__ off, long long* __restrict__ sums) {
    __shared__ long long part[1024];
    __shared__ int over[1024];
    const int t = threadIdx.x, T = blockDim.x;
    const int per = (n + T - 1) / T;
    const int b = t * per, e = min(n, b + per);
    long long s = 0;
    int ov = 0;
    for (int q = b; q < e; q++) {
        int v = nnz[q];
        s += v > 0 ? v : 0;
        ov += v == kOverflow;
    }
    part[t] = s;
    over[t] = ov;
    __syncthreads();
    for (int d = 1; d < T; d <<= 1) {
        long long x = t >= d ? part[t - d] : 0;
        int y = t >= d ? over[t - d] : 0;
        __syncthreads();
        part[t] += x;
        over[t] += y;
        __syncthreads();
    }
    long long run = part[t] - s;
    for (int q = b; q < e; q++) {
        off[q] = int(run);
        int v = nnz[q];
        run += v > 0 ? v : 0;
    }
    if (t == T - 1) {
        sums[0] = part[T - 1];
        sums[1] = over[T - 1];
    }
}

// A chunk's merged rows appended to the staging area at stage0 + their scanned offsets; each ray's
// place and size recorded under its global index.
__global__ void stage_kernel(const int* __restrict__ out_node, const float* __restrict__ out_len,
                             const int* __restrict__ nnz, const int* __restrict__ off,
                             const int64_t* __restrict__ rec_base, const int* __restrict__ ray_of, int nrays,
                             long long stage0, int* __restrict__ stage_col, float* __restrict__ stage_len,
                             long long* __restrict__ stage_off, int* __restrict__ ray_nnz) {
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int r = blockIdx.x * wpb + (threadIdx.x >> 5); r < nrays; r += gridDim.x * wpb) {
        const int c = nnz[r];
        const long long o = stage0 + off[r];
        if (lane == 0) {
            stage_off[ray_of[r]] = o;
            ray_nnz[ray_of[r]] = c;
        }
        const int64_t b = rec_base[r];
        for (int q = lane; q < c; q += 32) {
            stage_col[o + q] = out_node[b + q];
            stage_len[o + q] = out_len[b + q];
        }
    }
}

// Every row from the staging area into the CSR arrays in arrival order (row_ptr from the scan).
__global__ void emit_kernel(const int* __restrict__ stage_col, const float* __restrict__ stage_len,
                            const long long* __restrict__ stage_off, const int* __restrict__ ray_nnz,
                            const int* __restrict__ off, int nrays, int* __restrict__ row_ptr,
                            int* __restrict__ col, float* __restrict__ len, uint8_t* __restrict__ ok) {
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int r = blockIdx.x * wpb + (threadIdx.x >> 5); r < nrays; r += gridDim.x * wpb) {
        const int c = ray_nnz[r];
        const long long o = off[r];
        if (lane == 0) {
            row_ptr[r] = int(o);
            ok[r] = c >= 0 ? 1 : 0;
        }
        const long long s = stage_off[r];
        for (int q = lane; q < c; q += 32) {
            col[o + q] = stage_col[s + q];
            len[o + q] = stage_len[s + q];
        }
    }
}

RGrid make_rgrid(const host::Grid& g) {
    RGrid r{};
    r.nx = g.nx; r.ny = g.ny; r.nz = g.nz;
    r.min_lon = g.min_lon; r.min_lat = g.min_lat; r.min_dep = g.min_dep;
    r.dlon = g.dlon; r.dlat = g.dlat; r.ddep = g.ddep;
    r.dlon_rad = g.dlon_rad; r.dlat_rad = g.dlat_rad;
    r.centre_lon = g.centre_lon;
    r.lon_last = g.lon[g.nx - 1]; r.lat_last = g.lat[g.ny - 1]; r.dep_last = g.dep[g.nz - 1];
    r.min_spacing_km = g.min_spacing_km();
    return r;
}

}  // namespace rays
}  // namespace ts

using namespace ts;
using namespace ts::rays;

struct ts_rows {
    ts_ctx* ctx = nullptr;
    int n_rows = 0;
    int64_t nnz = 0;
    int* row_ptr = nullptr;   // device, n_rows + 1
    int* col = nullptr;       // device, nnz
    float* len = nullptr;
    double* tcg = nullptr;    // device, 4 per row
    uint8_t* ok = nullptr;
    double* outside = nullptr;  // device, per row: RayRow.OutsideTime
    // Stream-ordered frees: no device-wide synchronisation while other work runs (serving).
    ~ts_rows() {
        cudaStream_t s = ctx ? ctx->stream : nullptr;
        for (void* p : {static_cast<void*>(row_ptr), static_cast<void*>(col), static_cast<void*>(len),
                        static_cast<void*>(tcg), static_cast<void*>(ok), static_cast<void*>(outside)})
            if (p) cudaFreeAsync(p, s);
    }
};

namespace ts {
namespace rays {

static int trace_impl(ts_ctx* ctx, const host::Grid& fwd, const float* tables_dev, const float* const* table_ptrs_host,
                      int n_tables, const double* table_station_host, const host::Grid& inv, int n_rays,
                      const int32_t* table_of_host, const double* events_host, double step_km, ts_rows** out,
                      RayStats* st, const int32_t* table_phase_host) {
    cudaStream_t s = ctx->stream;
    const int64_t n = fwd.count();
    for (int a = 0; a < n_rays; a++)
        if (table_of_host[a] < 0 || table_of_host[a] >= n_tables) return ctx->fail(TS_E_ARG, "table_of out of range");
    if (!(step_km > 0)) return ctx->fail(TS_E_ARG, "step must be positive");
    if (fwd.variable || inv.variable) return ctx->fail(TS_E_ARG, "rays need uniform grids");
    // The result is freed on every early return; handed to the caller at the end.
    std::unique_ptr<ts_rows> rows_own(new ts_rows());
    ts_rows* rows = rows_own.get();
    rows->ctx = ctx;
    rows->n_rows = n_rays;
    auto bail = [&](int code) { return code; };
    if (ctx->alloc_async(&rows->row_ptr, sizeof(int) * (n_rays + 1), s) != cudaSuccess ||
        ctx->alloc_async(&rows->tcg, sizeof(double) * 4 * std::max(1, n_rays), s) != cudaSuccess ||
        ctx->alloc_async(&rows->ok, std::max(1, n_rays), s) != cudaSuccess ||
        ctx->alloc_async(&rows->outside, sizeof(double) * std::max(1, n_rays), s) !=
            cudaSuccess) {
        cudaGetLastError();
        ctx->fail(TS_E_NOMEM, "row buffers");
        return bail(TS_E_NOMEM);
    }
    TS_BUF(ctx, d_station, double, "rays.station", 3 * std::max(1, n_tables));
    TS_BUF(ctx, d_table_of, int, "rays.table_of", std::max(1, n_rays));
    TS_BUF(ctx, d_events, double, "rays.events", 3 * std::max(1, n_rays));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_station, table_station_host, sizeof(double) * 3 * n_tables, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_table_of, table_of_host, sizeof(int) * n_rays, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_events, events_host, sizeof(double) * 3 * n_rays, cudaMemcpyHostToDevice, s));

    TraceArgs a{};
    a.fwd = make_rgrid(fwd);
    a.inv = make_rgrid(inv);
    a.tables = tables_dev;
    a.table_n = n;
    a.table_ptr = nullptr;
    if (table_ptrs_host) {
        TS_BUF(ctx, d_ptrs, const float*, "rays.table_ptrs", std::max(1, n_tables));
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_ptrs, table_ptrs_host, sizeof(const float*) * n_tables,
                                         cudaMemcpyHostToDevice, s));
        a.table_ptr = d_ptrs;
    }
    a.table_station = d_station;
    a.table_of = d_table_of;
    a.events = d_events;
    a.step_km = step_km;
    a.piece_km = 0.5 * inv.min_spacing_km();  // RayTracing.cs:130
    a.tcg = rows->tcg;
    a.outside = rows->outside;
    TS_BUF(ctx, d_steps, unsigned long long, "rays.steps", 1);
    TS_CUDA_TRY(ctx, cudaMemsetAsync(d_steps, 0, sizeof(unsigned long long), s));
    a.steps = d_steps;
    // The extended domain's background (ts_set_background) and each table's phase.
    a.bg_n = ctx->bg_n;
    a.bg = a.bg_n > 0 ? static_cast<const double*>(ctx->buf("rays.background", sizeof(double) * 3 * a.bg_n))
                      : nullptr;
    std::vector<int32_t> phases(std::max(1, n_tables), 0);
    if (table_phase_host)
        for (int t = 0; t < n_tables; t++) phases[t] = table_phase_host[t] == 1 ? 1 : 0;
    TS_BUF(ctx, d_phase, int, "rays.table_phase", std::max(1, n_tables));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_phase, phases.data(), sizeof(int) * phases.size(), cudaMemcpyHostToDevice, s));
    a.table_phase = d_phase;

    const auto th0 = std::chrono::steady_clock::now();
    // Record room per ray: one record per node per inversion cell crossed, with room for a path
    // three times the straight length; a ray that needs more is traced again with four times the room.
    constexpr int kMaxCap = 16384;  // the larger merge pass sorts up to this many in 128 KB
    std::vector<int> cap_of(std::max(1, n_rays));
    {
        // The straight lengths on the host's threads (two trigonometric conversions per ray).
        auto room = [&](int q0, int q1) {
            for (int q = q0; q < q1; q++) {
                const double* ev = events_host + 3 * q;
                const double* stn = table_station_host + 3 * table_of_host[q];
                const double d =
                    host::dist(host::to_cartesian(ev[0], ev[1], ev[2]), host::to_cartesian(stn[0], stn[1], stn[2]));
                cap_of[q] = int(std::min(double(kMaxCap), 8.0 * (3.0 * d / a.piece_km + 32)));
            }
        };
        const int nt = n_rays < 65536 ? 1 : int(std::min(16u, std::max(1u, std::thread::hardware_concurrency())));
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; t++)
            pool.emplace_back(room, int(int64_t(n_rays) * t / nt), int(int64_t(n_rays) * (t + 1) / nt));
        room(0, int(int64_t(n_rays) / nt));
        for (auto& th : pool) th.join();
    }
    // Rays in order of their table (a counting sort, stable): a chunk's rays read few tables, which
    // stay in L2.
    std::vector<int> order(n_rays);
    {
        std::vector<int> at(n_tables + 1, 0);
        for (int q = 0; q < n_rays; q++) at[table_of_host[q] + 1]++;
        for (int t = 0; t < n_tables; t++) at[t + 1] += at[t];
        for (int q = 0; q < n_rays; q++) order[at[table_of_host[q]]++] = q;
    }
    const auto th1 = std::chrono::steady_clock::now();
    // Chunk budget: record slots (12 B of record + 8 B of merged output each) of two chunks in
    // flight within a share of the free device memory, at most 400 M slots per chunk. A call whose
    // rooms all fit in 16 M slots (320 MB) is one chunk without asking for the free memory, which
    // costs milliseconds per query while other work holds the device (small calls, serving).
    int64_t need = 0;
    for (int q = 0; q < n_rays; q++) need += cap_of[q];
    int64_t budget = std::max<int64_t>(need, 1);
    if (need > (int64_t(16) << 20)) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        cudaGetLastError();
        budget = std::max<int64_t>(int64_t(kMaxCap) * 64,
                                   std::min<int64_t>(int64_t(400) << 20, int64_t(free_b / 8 / 20)));
    }
    TS_BUF(ctx, ray_nnz, int, "rays.ray_nnz", std::max(1, n_rays));
    TS_BUF(ctx, stage_off, long long, "rays.stage_off", std::max(1, n_rays));
    // The staging area (rows in chunk order), freed on every return.
    struct Stage {
        cudaStream_t s;
        int* col = nullptr;
        float* len = nullptr;
        void free() {
            if (col) cudaFreeAsync(col, s);
            if (len) cudaFreeAsync(len, s);
            col = nullptr;
            len = nullptr;
        }
        ~Stage() { free(); }
    } stage{s};
    int*& stage_col = stage.col;
    float*& stage_len = stage.len;
    int64_t stage_cap = 0, stage_used = 0;
    auto free_stage = [&]() { stage.free(); };
    // Two chunks in flight: while the device traces chunk k, the host reads chunk k−1's row total and
    // queues its staging copy behind it, so the stream never waits on the host.
    struct Events {
        cudaEvent_t e[2] = {nullptr, nullptr};
        Events() {
            for (auto& x : e) cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
        }
        ~Events() {
            for (auto& x : e) cudaEventDestroy(x);
        }
    } done;
    long long* h_sums = static_cast<long long*>(ctx->host_buf("rays.sums_h", sizeof(long long) * 4));
    if (!h_sums) return bail(TS_E_NOMEM);
    EventPair ev;
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    cudaEventRecord(e0, s);
    std::vector<int> pending = order;
    for (int pass = 0; !pending.empty(); pass++) {
        // The pass's chunks: rays in order while their rooms fit the budget; each ray's room and
        // place, for every chunk, copied to the device at once.
        struct Chunk {
            size_t c0, c1;
            int64_t used;
            int maxcap;
        };
        std::vector<Chunk> chunks;
        const size_t np = pending.size();
        int* h_ray = static_cast<int*>(ctx->host_buf("rays.plan_ray", sizeof(int) * np));
        int64_t* h_base = static_cast<int64_t*>(ctx->host_buf("rays.plan_base", sizeof(int64_t) * np));
        int* h_cap = static_cast<int*>(ctx->host_buf("rays.plan_cap", sizeof(int) * np));
        if (!h_ray || !h_base || !h_cap) return bail(TS_E_NOMEM);
        int64_t max_used = 1;
        int max_nr = 1, maxcap_all = 32;
        for (size_t c0 = 0; c0 < np;) {
            Chunk c{c0, c0, 0, 32};
            while (c.c1 < np && (c.c1 == c0 || c.used + cap_of[pending[c.c1]] <= budget) &&
                   c.c1 - c0 < (size_t(1) << 20)) {
                const int q = pending[c.c1];
                h_ray[c.c1] = q;
                h_base[c.c1] = c.used;
                h_cap[c.c1] = cap_of[q];
                c.used += cap_of[q];
                c.maxcap = std::max(c.maxcap, cap_of[q]);
                c.c1++;
            }
            max_used = std::max(max_used, c.used);
            max_nr = std::max(max_nr, int(c.c1 - c0));
            maxcap_all = std::max(maxcap_all, c.maxcap);
            chunks.push_back(c);
            c0 = c.c1;
        }
        TS_BUF(ctx, d_ray_of, int, "rays.ray_of", np);
        TS_BUF(ctx, d_base, int64_t, "rays.rec_base", np);
        TS_BUF(ctx, d_cap, int, "rays.rec_cap", np);
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_ray_of, h_ray, sizeof(int) * np, cudaMemcpyHostToDevice, s));
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_base, h_base, sizeof(int64_t) * np, cudaMemcpyHostToDevice, s));
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_cap, h_cap, sizeof(int) * np, cudaMemcpyHostToDevice, s));
        // Per set of a chunk in flight: records, merged rows, row sizes and offsets, the two totals.
        struct Set {
            int *rec_node, *rec_count, *out_node, *nnz, *off;
            double* rec_val;
            float* out_len;
            long long* sums;
        } set[2];
        for (int b = 0; b < 2; b++) {
            const std::string k = b ? "1" : "0";
            set[b].rec_node = static_cast<int*>(ctx->buf("rays.rec_node" + k, sizeof(int) * size_t(max_used)));
            set[b].rec_val = static_cast<double*>(ctx->buf("rays.rec_val" + k, sizeof(double) * size_t(max_used)));
            set[b].out_node = static_cast<int*>(ctx->buf("rays.out_node" + k, sizeof(int) * size_t(max_used)));
            set[b].out_len = static_cast<float*>(ctx->buf("rays.out_len" + k, sizeof(float) * size_t(max_used)));
            set[b].rec_count = static_cast<int*>(ctx->buf("rays.rec_count" + k, sizeof(int) * max_nr));
            set[b].nnz = static_cast<int*>(ctx->buf("rays.nnz" + k, sizeof(int) * max_nr));
            set[b].off = static_cast<int*>(ctx->buf("rays.off" + k, sizeof(int) * max_nr));
            set[b].sums = static_cast<long long*>(ctx->buf("rays.sums" + k, sizeof(long long) * 2));
            if (!set[b].rec_node || !set[b].rec_val || !set[b].out_node || !set[b].out_len || !set[b].rec_count ||
                !set[b].nnz || !set[b].off || !set[b].sums)
                return bail(TS_E_NOMEM);
        }
        // Small sort size for most rays; the rest in a second pass with one warp per block.
        const int Psmall = 2048, W = 4;
        int Pbig_all = Psmall;
        while (Pbig_all < maxcap_all) Pbig_all <<= 1;
        TS_CUDA_TRY(ctx, cudaFuncSetAttribute(merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              std::max(W * Psmall, Pbig_all) * 8));
        std::vector<int> retry;
        auto launch = [&](size_t k) -> int {
            const Chunk& c = chunks[k];
            const Set& z = set[k & 1];
            const int nr = int(c.c1 - c.c0);
            if (st) st->chunks++;
            a.ray_of = d_ray_of + c.c0;
            a.nrays = nr;
            a.rec_base = d_base + c.c0;
            a.rec_cap = d_cap + c.c0;
            a.rec_node = z.rec_node;
            a.rec_val = z.rec_val;
            a.rec_count = z.rec_count;
            if (n_rays <= ctx->ray_warp_max) trace_warp_kernel<<<(nr + 3) / 4, 128, 0, s>>>(a);
            else trace_kernel<<<(nr + 127) / 128, 128, 0, s>>>(a);
            TS_CUDA_TRY(ctx, cudaGetLastError());
            int Pbig = Psmall;
            while (Pbig < c.maxcap) Pbig <<= 1;
            merge_kernel<<<std::min((nr + W - 1) / W, ctx->sm_count * 8), W * 32, size_t(W) * Psmall * 8, s>>>(
                z.rec_node, z.rec_val, z.rec_count, d_base + c.c0, nr, Psmall, 0, z.out_node, z.out_len, z.nnz);
            TS_CUDA_TRY(ctx, cudaGetLastError());
            if (Pbig > Psmall) {
                merge_kernel<<<std::min(nr, ctx->sm_count * 2), 32, size_t(Pbig) * 8, s>>>(
                    z.rec_node, z.rec_val, z.rec_count, d_base + c.c0, nr, Pbig, Psmall, z.out_node, z.out_len, z.nnz);
                TS_CUDA_TRY(ctx, cudaGetLastError());
            }
            scan_kernel<<<1, 1024, 0, s>>>(z.nnz, nr, z.off, z.sums);
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(h_sums + 2 * (k & 1), z.sums, sizeof(long long) * 2,
                                             cudaMemcpyDeviceToHost, s));
            TS_CUDA_TRY(ctx, cudaEventRecord(done.e[k & 1], s));
            return TS_OK;
        };
        auto finish = [&](size_t k) -> int {
            const Chunk& c = chunks[k];
            const Set& z = set[k & 1];
            const int nr = int(c.c1 - c.c0);
            TS_CUDA_TRY(ctx, cudaEventSynchronize(done.e[k & 1]));
            const long long tot = h_sums[2 * (k & 1)], over = h_sums[2 * (k & 1) + 1];
            if (over > 0) {
                // Rays that ran out of room: traced again later with four times the room. (The set's
                // sizes are not overwritten before this chunk's staging copy below.)
                std::vector<int> hn(nr);
                TS_CUDA_TRY(ctx, cudaMemcpyAsync(hn.data(), z.nnz, sizeof(int) * nr, cudaMemcpyDeviceToHost, s));
                TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
                for (int r = 0; r < nr; r++) {
                    if (hn[r] != kOverflow) continue;
                    const int q = pending[c.c0 + r];
                    if (cap_of[q] >= kMaxCap)
                        return ctx->fail(TS_E_CAPACITY, "a ray needs more records than supported");
                    cap_of[q] = std::min(kMaxCap, cap_of[q] * 4);
                    retry.push_back(q);
                }
                if (st) st->retraced_chunks++;
            }
            if (stage_used + tot > stage_cap) {
                const int64_t want = std::max<int64_t>({stage_used + tot, stage_cap * 2, 1024});
                int* ncol = nullptr;
                float* nlen = nullptr;
                if (ctx->alloc_async(&ncol, sizeof(int) * want, s) != cudaSuccess ||
                    ctx->alloc_async(&nlen, sizeof(float) * want, s) != cudaSuccess) {
                    cudaGetLastError();
                    if (ncol) cudaFreeAsync(ncol, s);
                    return ctx->fail(TS_E_NOMEM, "row staging arrays");
                }
                if (stage_used > 0) {
                    cudaMemcpyAsync(ncol, stage_col, sizeof(int) * stage_used, cudaMemcpyDeviceToDevice, s);
                    cudaMemcpyAsync(nlen, stage_len, sizeof(float) * stage_used, cudaMemcpyDeviceToDevice, s);
                }
                free_stage();
                stage_col = ncol;
                stage_len = nlen;
                stage_cap = want;
            }
            stage_kernel<<<std::min((nr + 7) / 8, ctx->sm_count * 16), 256, 0, s>>>(
                z.out_node, z.out_len, z.nnz, z.off, d_base + c.c0, d_ray_of + c.c0, nr, stage_used, stage_col,
                stage_len, stage_off, ray_nnz);
            TS_CUDA_TRY(ctx, cudaGetLastError());
            stage_used += tot;
            return TS_OK;
        };
        for (size_t k = 0; k < chunks.size(); k++) {
            int rc = launch(k);
            if (rc == TS_OK && k > 0) rc = finish(k - 1);
            if (rc != TS_OK) return bail(rc);
        }
        if (!chunks.empty()) {
            const int rc = finish(chunks.size() - 1);
            if (rc != TS_OK) return bail(rc);
        }
        pending.swap(retry);
    }
    // Rows in arrival order: offsets of every ray's row, then the copy into the CSR arrays.
    int64_t total = 0;
    if (n_rays > 0) {
        TS_BUF(ctx, off_all, int, "rays.off_all", n_rays);
        TS_BUF(ctx, sums_all, long long, "rays.sums_all", 2);
        scan_kernel<<<1, 1024, 0, s>>>(ray_nnz, n_rays, off_all, sums_all);
        long long h[2] = {0, 0};
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(h, sums_all, sizeof h, cudaMemcpyDeviceToHost, s));
        TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        total = h[0];
        if (total > INT32_MAX) {
            free_stage();
            return bail(ctx->fail(TS_E_CAPACITY, "more than 2^31 non-zeros"));
        }
        const int64_t alloc = std::max<int64_t>(1, total);
        if (ctx->alloc_async(&rows->col, sizeof(int) * alloc, s) != cudaSuccess ||
            ctx->alloc_async(&rows->len, sizeof(float) * alloc, s) != cudaSuccess) {
            cudaGetLastError();
            free_stage();
            return bail(ctx->fail(TS_E_NOMEM, "CSR arrays"));
        }
        emit_kernel<<<std::min((n_rays + 7) / 8, ctx->sm_count * 16), 256, 0, s>>>(
            stage_col, stage_len, stage_off, ray_nnz, off_all, n_rays, rows->row_ptr, rows->col, rows->len,
            rows->ok);
        TS_CUDA_TRY(ctx, cudaGetLastError());
    }
    free_stage();
    int tot32 = int(total);
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(rows->row_ptr + n_rays, &tot32, sizeof(int), cudaMemcpyHostToDevice, s));
    cudaEventRecord(e1, s);
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    rows->nnz = total;
    unsigned long long h_steps = 0;
    TS_CUDA_TRY(ctx, cudaMemcpy(&h_steps, d_steps, sizeof h_steps, cudaMemcpyDeviceToHost));
    if (st) {
        st->steps += h_steps;
        st->device_ms += ms;
        st->setup_ms += std::chrono::duration<double, std::milli>(th1 - th0).count();
        st->wall_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - th0).count();
    }
    *out = rows_own.release();
    return TS_OK;
}

}  // namespace rays
}  // namespace ts

namespace ts {
namespace rays {

int trace_on_device(ts_ctx* ctx, const host::Grid& fwd, const float* tables_dev, int n_tables,
                    const double* table_station_host, const host::Grid& inv, int n_rays, const int32_t* table_of_host,
                    const double* events_host, double step_km, ts_rows** out, RayStats* st,
                    const int32_t* table_phase_host) {
    return trace_impl(ctx, fwd, tables_dev, nullptr, n_tables, table_station_host, inv, n_rays, table_of_host,
                      events_host, step_km, out, st, table_phase_host);
}

int trace_on_device(ts_ctx* ctx, const host::Grid& fwd, const std::vector<const float*>& tables, const double* table_station_host,
                    const host::Grid& inv, int n_rays, const int32_t* table_of_host, const double* events_host,
                    double step_km, ts_rows** out, RayStats* st, const int32_t* table_phase_host) {
    return trace_impl(ctx, fwd, nullptr, tables.data(), int(tables.size()), table_station_host, inv, n_rays,
                      table_of_host, events_host, step_km, out, st, table_phase_host);
}

int split_rows(ts_ctx* ctx, const ts_rows* all, const std::vector<int>& row_begin, std::vector<ts_rows*>& parts) {
    cudaStream_t s = ctx->stream;
    std::vector<int> rp(all->n_rows + 1);
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(rp.data(), all->row_ptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost, s));
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    parts.assign(row_begin.size() - 1, nullptr);
    for (size_t k = 0; k + 1 < row_begin.size(); k++) {
        const int r0 = row_begin[k], r1 = row_begin[k + 1], n = r1 - r0;
        const int64_t z0 = rp[r0], nnz = int64_t(rp[r1]) - rp[r0];
        auto* p = new ts_rows();
        p->ctx = ctx;
        p->n_rows = n;
        p->nnz = nnz;
        std::vector<int> local(n + 1);
        for (int q = 0; q <= n; q++) local[q] = int(rp[r0 + q] - z0);
        auto fail = [&]() {
            cudaGetLastError();
            delete p;
            for (auto*& q : parts) {
                delete q;
                q = nullptr;
            }
            return ctx->fail(TS_E_NOMEM, "row buffers");
        };
        if (ctx->alloc_async(&p->row_ptr, sizeof(int) * (n + 1), s) != cudaSuccess ||
            ctx->alloc_async(&p->tcg, sizeof(double) * 4 * std::max(1, n), s) != cudaSuccess ||
            ctx->alloc_async(&p->ok, std::max(1, n), s) != cudaSuccess ||
            ctx->alloc_async(&p->outside, sizeof(double) * std::max(1, n), s) != cudaSuccess ||
            ctx->alloc_async(&p->col, sizeof(int) * std::max<int64_t>(1, nnz), s) != cudaSuccess ||
            ctx->alloc_async(&p->len, sizeof(float) * std::max<int64_t>(1, nnz), s) != cudaSuccess)
            return fail();
        // From pageable memory the copy has taken the source when the call returns.
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(p->row_ptr, local.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
        if (n) {
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(p->tcg, all->tcg + 4 * int64_t(r0), sizeof(double) * 4 * n,
                                             cudaMemcpyDeviceToDevice, s));
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(p->ok, all->ok + r0, size_t(n), cudaMemcpyDeviceToDevice, s));
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(p->outside, all->outside + r0, sizeof(double) * n,
                                             cudaMemcpyDeviceToDevice, s));
        }
        if (nnz) {
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(p->col, all->col + z0, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(p->len, all->len + z0, sizeof(float) * nnz, cudaMemcpyDeviceToDevice, s));
        }
        parts[k] = p;
    }
    return TS_OK;
}

void free_rows(ts_rows* rows) { delete rows; }

void rows_view(const ts_rows* rows, int* n_rows, int64_t* nnz, const int** row_ptr, const int** col, const float** len) {
    *n_rows = rows->n_rows;
    *nnz = rows->nnz;
    *row_ptr = rows->row_ptr;
    *col = rows->col;
    *len = rows->len;
}

}  // namespace rays
}  // namespace ts

extern "C" {

int ts_rays_set_warp_max(ts_ctx* ctx, int32_t max_rays) {
    if (!ctx || max_rays < 0) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    ctx->ray_warp_max = max_rays;
    return TS_OK;
}

int ts_rays_trace(ts_ctx* ctx, const ts_grid* fwd, int32_t n_tables, const float* tables, const double* table_station,
                  const ts_grid* inv, int32_t n_rays, const int32_t* table_of, const double* events, double step_km,
                  ts_rows** out) {
    if (!ctx || !out) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = nullptr;
    if (!fwd || !inv || host::Grid::validate(*fwd) || host::Grid::validate(*inv))
        return ctx->fail(TS_E_ARG, "invalid grid");
    if (n_tables <= 0 || n_rays < 0 || !tables || !table_station || (n_rays > 0 && (!table_of || !events)))
        return ctx->fail(TS_E_ARG, "null array or empty table set");
    host::Grid gf(*fwd), gi(*inv);
    const size_t bytes = sizeof(float) * size_t(n_tables) * size_t(gf.count());
    float* d_tables = static_cast<float*>(ctx->buf("rays.tables", bytes));
    if (!d_tables) return TS_E_NOMEM;
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_tables, tables, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return ts::rays::trace_on_device(ctx, gf, d_tables, n_tables, table_station, gi, n_rays, table_of, events, step_km,
                                     out, nullptr);
}

int ts_rows_info(ts_rows* rows, int32_t* n_rows, int64_t* nnz) {
    if (!rows) return TS_E_ARG;
    if (n_rows) *n_rows = rows->n_rows;
    if (nnz) *nnz = rows->nnz;
    return TS_OK;
}

int ts_rows_copy(ts_rows* rows, int32_t* row_ptr, int32_t* col, float* len, double* tcalc_grad, uint8_t* ok) {
    if (!rows) return TS_E_ARG;
    ts_ctx* ctx = rows->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int n = rows->n_rows;
    if (row_ptr) TS_CUDA_TRY(ctx, cudaMemcpyAsync(row_ptr, rows->row_ptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    if (col && rows->nnz) TS_CUDA_TRY(ctx, cudaMemcpyAsync(col, rows->col, sizeof(int) * rows->nnz, cudaMemcpyDeviceToHost, s));
    if (len && rows->nnz) TS_CUDA_TRY(ctx, cudaMemcpyAsync(len, rows->len, sizeof(float) * rows->nnz, cudaMemcpyDeviceToHost, s));
    if (tcalc_grad && n) TS_CUDA_TRY(ctx, cudaMemcpyAsync(tcalc_grad, rows->tcg, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s));
    if (ok && n) TS_CUDA_TRY(ctx, cudaMemcpyAsync(ok, rows->ok, size_t(n), cudaMemcpyDeviceToHost, s));
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    return TS_OK;
}

int ts_rows_outside(ts_rows* rows, double* outside) {
    if (!rows || !outside) return TS_E_ARG;
    ts_ctx* ctx = rows->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (rows->n_rows > 0)
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(outside, rows->outside, sizeof(double) * rows->n_rows, cudaMemcpyDeviceToHost,
                                         ctx->stream));
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return TS_OK;
}

void ts_rows_free(ts_rows* rows) {
    if (!rows) return;
    std::lock_guard<std::recursive_mutex> lk(rows->ctx->mu);
    cudaSetDevice(rows->ctx->device);
    delete rows;
}

}  // extern "C"
