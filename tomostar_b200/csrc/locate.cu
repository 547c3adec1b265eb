// Event location on travel-time tables kept on the device: EventLocator.Locate
// (Location/EventLocator.cs:59-104) for many events at once, as Relocation.Absolute runs it
// (Location/Relocation.cs:76-91).
//
// Per round (at most three): the grid search (EventLocator.cs:107-163) as one thread per candidate
// node, so that the reads of one table by a warp's consecutive candidates coalesce; each candidate's
// residuals are put in order by a stable insertion sort for the weighted-median origin time
// (:297-309) and every sum is taken in the reference's order, so the best node and its origin time
// equal the sequential search's. Then Geiger's Levenberg-Marquardt iterations (:166-256) and the
// outlier rule (:84-90) as one warp per event: lanes evaluate observations (trilinear time and
// gradient on the float32 tables) and every lane forms the normal equations in observation order
// from the lanes' values, so all lanes hold the same sums and decisions.
//
// The file is compiled with -fmad=false: each product and sum rounds on its own, as .NET's does.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "geo_dev.cuh"
#include "host_geo.h"
#include "tables.h"

namespace ts {
namespace rays {
geo::RGrid make_rgrid(const host::Grid& g);
}

namespace loc {

using geo::RGrid;

constexpr int kSearchThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

// One observation as the kernels read it: its table, pick time, weight and station correction.
struct ObsD {
    const float* tb;
    double sec, w, corr;
};

// One box search of one event (EventLocator.Search, :143-163): stride lattice from (i0, j0, k0)
// with ci x cj x ck candidates, scanned k outermost, i innermost.
struct SearchTask {
    int event, i0, j0, k0, stride, ci, cj, ck, count, block0;
};

struct Partial {
    double m;
    int c, pad;
};

// Per-event state between the stages.
struct EvState {
    double slon, slat, sdep;                   // the catalogue location (the search's start)
    double lon, lat, dep, t0;                  // grid-search result, then Geiger's
    double rms, eh, emin, eaz, edep, et;       // Hypocentre's Rms and errors
    int best, nused, rejected, iterations, done, located;
};

struct Params {
    int max_it, min_phases, fix_depth, pad;
    double damping, outlier_mads, outlier_floor;
};

__device__ __forceinline__ double dnan() { return __longlong_as_double(0x7ff8000000000000LL); }

// GridSearch's Misfit (EventLocator.cs:111-124) at node idx over o[0..n): residuals, their stable
// order, the weighted median t0 and the weighted L1 misfit. r and si are the thread's scratch.
template <int NMAX>
__device__ double node_misfit(const ObsD* o, int n, int64_t idx, double& t0) {
    double r[NMAX];
    unsigned short si[NMAX];
    int np = 0;
    for (int q = 0; q < n; q++) {
        const float t = __ldg(o[q].tb + idx);
        if (isfinite(t)) {
            const double v = o[q].sec - double(t) - o[q].corr;
            r[q] = v;
            int p = np++;
            while (p > 0 && r[si[p - 1]] > v) {
                si[p] = si[p - 1];
                p--;
            }
            si[p] = (unsigned short)q;
        } else {
            r[q] = dnan();
        }
    }
    t0 = 0;
    if (np > 0) {
        double sum = 0;
        for (int p = 0; p < np; p++) sum += o[si[p]].w;
        const double half = sum / 2;
        double acc = 0;
        t0 = r[si[np - 1]];
        for (int p = 0; p < np; p++) {
            acc += o[si[p]].w;
            if (acc >= half) {
                t0 = r[si[p]];
                break;
            }
        }
    }
    double m = 0;
    for (int q = 0; q < n; q++) m += isnan(r[q]) ? 10 * o[q].w : o[q].w * fabs(r[q] - t0);
    return m;
}

__device__ __forceinline__ bool better(double m1, int c1, double m2, int c2) {
    return m1 < m2 || (m1 == m2 && c1 < c2);
}

// The task of a block: the last one whose first block is not after it.
__device__ __forceinline__ int task_of_block(const SearchTask* tasks, int n_tasks) {
    int lo = 0, hi = n_tasks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].block0 <= int(blockIdx.x)) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int64_t candidate_node(const SearchTask& t, int c, int nx, int ny) {
    const int ii = t.i0 + (c % t.ci) * t.stride;
    const int jj = t.j0 + ((c / t.ci) % t.cj) * t.stride;
    const int kk = t.k0 + (c / (t.ci * t.cj)) * t.stride;
    return (int64_t(kk) * ny + jj) * nx + ii;
}

// Block-wide first minimum of (m, c) over 256 threads; thread 0 writes the block's partial.
__device__ __forceinline__ void block_best(double m, int cc, Partial* partial) {
    __shared__ double wm[kSearchThreads / 32];
    __shared__ int wc[kSearchThreads / 32];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const double m2 = __shfl_down_sync(kFull, m, d);
        const int c2 = __shfl_down_sync(kFull, cc, d);
        if (better(m2, c2, m, cc)) {
            m = m2;
            cc = c2;
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        wm[warp] = m;
        wc[warp] = cc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bm = wm[0];
        int bc = wc[0];
        for (int w = 1; w < kSearchThreads / 32; w++)
            if (better(wm[w], wc[w], bm, bc)) {
                bm = wm[w];
                bc = wc[w];
            }
        partial[blockIdx.x] = Partial{bm, bc, 0};
    }
}

// Exact path, any weights and up to 1024 picks: one thread per candidate, the residuals ordered by a
// stable insertion sort and every sum taken in the reference's order.
template <int NMAX>
__global__ void __launch_bounds__(kSearchThreads) search_kernel(const SearchTask* __restrict__ tasks, int n_tasks,
                                                                const int* __restrict__ off,
                                                                const EvState* __restrict__ st,
                                                                const ObsD* __restrict__ olist, int nx, int ny,
                                                                Partial* __restrict__ partial) {
    __shared__ ObsD so[NMAX];
    const SearchTask t = tasks[task_of_block(tasks, n_tasks)];
    const int n = st[t.event].nused;
    for (int q = threadIdx.x; q < n; q += blockDim.x) so[q] = olist[off[t.event] + q];
    __syncthreads();
    const int c = (int(blockIdx.x) - t.block0) * kSearchThreads + threadIdx.x;
    double m = dinf();
    int cc = 0x7fffffff;
    if (c < t.count) {
        double t0;
        m = node_misfit<NMAX>(so, n, candidate_node(t, c, nx, ny), t0);
        cc = c;
    }
    block_best(m, cc, partial);
}

// Bitonic sort of 32*E (key, pick) pairs held E per lane (element j*32 + lane in slot j), ascending by
// key then pick: a total order, so the result is the stable sort by key.
template <int E>
__device__ __forceinline__ void warp_bitonic(double (&key)[E], int (&q)[E], int lane) {
    constexpr int N = 32 * E;
#pragma unroll
    for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
        for (int d = k >> 1; d > 0; d >>= 1) {
            if (d >= 32) {
#pragma unroll
                for (int j = 0; j < E; j++) {
                    const int jp = j ^ (d >> 5);
                    if (jp > j) {
                        const bool up = (((j * 32 + lane) & k) == 0);
                        const bool gt = key[j] > key[jp] || (key[j] == key[jp] && q[j] > q[jp]);
                        if (gt == up) {
                            const double tk = key[j];
                            key[j] = key[jp];
                            key[jp] = tk;
                            const int tq = q[j];
                            q[j] = q[jp];
                            q[jp] = tq;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < E; j++) {
                    const double ok = __shfl_xor_sync(kFull, key[j], d);
                    const int oq = __shfl_xor_sync(kFull, q[j], d);
                    const bool up = (((j * 32 + lane) & k) == 0);
                    const bool lower = (lane & d) == 0;
                    const bool gt = key[j] > ok || (key[j] == ok && q[j] > oq);
                    if (lower ? (gt == up) : (gt != up)) {
                        key[j] = ok;
                        q[j] = oq;
                    }
                }
            }
        }
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFull, v, d);
    return v;
}

// GridSearch's Misfit at one node by one warp, for dyadic non-negative weights (sums of at most 128
// of them are exact in any order): the weighted-median origin time exactly as the reference's, and
// the misfit either as a tree sum (fast) or in pick order (exact, the reference's rounding).
template <int E>
__device__ double warp_node_misfit(const ObsD* so, int n, int64_t idx, int lane, bool exact) {
    double key[E], r0[E], w0[E];
    int q[E];
#pragma unroll
    for (int j = 0; j < E; j++) {
        const int qq = j * 32 + lane;
        r0[j] = dnan();
        w0[j] = 0;
        key[j] = dinf();
        q[j] = 1024 + qq;  // padding sorts after every pick
        if (qq < n) {
            const float t = __ldg(so[qq].tb + idx);
            w0[j] = so[qq].w;
            q[j] = qq;
            if (isfinite(t)) {
                r0[j] = so[qq].sec - double(t) - so[qq].corr;
                key[j] = r0[j];
            }
        }
    }
    warp_bitonic<E>(key, q, lane);
    // Weights in sorted order (finite residuals only), their total and inclusive prefix sums.
    double ws[E];
    double total = 0;
#pragma unroll
    for (int j = 0; j < E; j++) {
        ws[j] = (key[j] < dinf()) ? so[q[j]].w : 0.0;
        total += ws[j];
    }
    total = warp_sum(total);
    const double half = total / 2;
    const unsigned finite0 = __ballot_sync(kFull, key[0] < dinf());
    double t0 = 0;
    if (finite0 != 0) {
        double carry = 0;
        bool found = false;
        double last = 0;
#pragma unroll
        for (int j = 0; j < E; j++) {
            double x = ws[j];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const double y = __shfl_up_sync(kFull, x, d);
                if (lane >= d) x += y;
            }
            const double acc = carry + x;
            carry += __shfl_sync(kFull, x, 31);
            const unsigned fin = __ballot_sync(kFull, key[j] < dinf());
            if (fin) last = __shfl_sync(kFull, key[j], 31 - __clz(fin));
            const unsigned hit = __ballot_sync(kFull, key[j] < dinf() && acc >= half);
            if (!found && hit) {
                t0 = __shfl_sync(kFull, key[j], __ffs(hit) - 1);
                found = true;
            }
        }
        if (!found) t0 = last;
    }
    double term[E];
    double m = 0;
#pragma unroll
    for (int j = 0; j < E; j++) {
        term[j] = (j * 32 + lane < n) ? (isnan(r0[j]) ? 10 * w0[j] : w0[j] * fabs(r0[j] - t0)) : 0.0;
        m += term[j];
    }
    if (!exact) return warp_sum(m);
    m = 0;
#pragma unroll
    for (int j = 0; j < E; j++)
        for (int l = 0; l < 32 && j * 32 + l < n; l++) m += __shfl_sync(kFull, term[j], l);
    return m;
}

// Fast path: one warp per candidate, kWarpCands consecutive candidates per warp. Each block then
// re-sums in pick order the candidates whose tree-summed misfit lies within 1e-12 (relative) of the
// block's smallest, which holds every candidate that can be the block's exact first minimum (two
// summation orders of n non-negative terms differ by at most 2(n-1)u of the sum), and reports the
// exact first minimum among them.
constexpr int kWarpCands = 8;
constexpr int kBlockCands = kWarpCands * (kSearchThreads / 32);

template <int E>
__global__ void __launch_bounds__(kSearchThreads, 4) search_warp_kernel(const SearchTask* __restrict__ tasks,
                                                                     int n_tasks, const int* __restrict__ off,
                                                                     const EvState* __restrict__ st,
                                                                     const ObsD* __restrict__ olist, int nx, int ny,
                                                                     Partial* __restrict__ partial) {
    __shared__ ObsD so[32 * E];
    __shared__ double fm[kBlockCands];
    __shared__ double fmin_s;
    const SearchTask t = tasks[task_of_block(tasks, n_tasks)];
    const int n = st[t.event].nused;
    for (int q = threadIdx.x; q < n; q += blockDim.x) so[q] = olist[off[t.event] + q];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cb = (int(blockIdx.x) - t.block0) * kBlockCands;
    for (int k = 0; k < kWarpCands; k++) {
        const int slot = warp * kWarpCands + k;
        const int c = cb + slot;
        double m = dinf();
        if (c < t.count) m = warp_node_misfit<E>(so, n, candidate_node(t, c, nx, ny), lane, false);
        if (lane == 0) fm[slot] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = fm[0];
        for (int i = 1; i < kBlockCands; i++) b = fmin(b, fm[i]);
        fmin_s = b;
    }
    __syncthreads();
    const double band = fmin_s + fmin_s * 1e-12;
    double best = dinf();
    int bc = 0x7fffffff;
    for (int k = 0; k < kWarpCands; k++) {
        const int slot = warp * kWarpCands + k;
        const int c = cb + slot;
        if (c >= t.count || !(fm[slot] <= band)) continue;
        const double m = warp_node_misfit<E>(so, n, candidate_node(t, c, nx, ny), lane, true);
        if (m < best || bc == 0x7fffffff) {
            best = m;
            bc = c;
        }
    }
    if (fmin_s == dinf()) {  // every misfit +inf: the first candidate stands for the block
        best = dinf();
        bc = cb;
    }
    // Warp 0's lane 0 of each warp holds that warp's exact best; reduce over warps.
    block_best(lane == 0 ? best : dinf(), lane == 0 ? bc : 0x7fffffff, partial);
}

// The best candidate of each task over its blocks (first minimum in scan order; every misfit +inf
// gives the first candidate, as Search returns Index(i0, j0, k0)), its node, origin time and place.
template <int NMAX>
__global__ void pick_best(const RGrid g, const SearchTask* __restrict__ tasks, int n_tasks,
                          const Partial* __restrict__ partial, const int* __restrict__ off,
                          const ObsD* __restrict__ olist, EvState* __restrict__ st, int fix_depth, int per_block,
                          int* __restrict__ best_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_tasks) return;
    const SearchTask t = tasks[k];
    const int nb = (t.count + per_block - 1) / per_block;
    double bm = partial[t.block0].m;
    int bc = partial[t.block0].c;
    for (int b = 1; b < nb; b++)
        if (partial[t.block0 + b].m < bm) {
            bm = partial[t.block0 + b].m;
            bc = partial[t.block0 + b].c;
        }
    if (!(bm < dinf())) bc = 0;
    const int ii = t.i0 + (bc % t.ci) * t.stride;
    const int jj = t.j0 + ((bc / t.ci) % t.cj) * t.stride;
    const int kk = t.k0 + (bc / (t.ci * t.cj)) * t.stride;
    const int64_t idx = (int64_t(kk) * g.ny + jj) * g.nx + ii;
    EvState& s = st[t.event];
    double t0;
    node_misfit<NMAX>(olist + off[t.event], s.nused, idx, t0);
    s.best = int(idx);
    s.lon = g.min_lon + ii * g.dlon;
    s.lat = g.min_lat + jj * g.dlat;
    s.dep = fix_depth ? s.sdep : g.min_dep + kk * g.ddep;
    s.t0 = t0;
    best_out[k] = int(idx);
}

// Math.Max and Math.Clamp of .NET (NaN propagates; Max prefers +0 over -0).
__device__ __forceinline__ double net_max(double a, double b) {
    if (isnan(a) || isnan(b)) return dnan();
    if (a == b) return signbit(a) ? b : a;
    return a > b ? a : b;
}
__device__ __forceinline__ double net_clamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

// DateTime.AddSeconds then TimeSpan.TotalSeconds: t0 truncated to 100 ns ticks, then ticks / 1e7.
__host__ __device__ __forceinline__ double tick_seconds(double t0) {
    const double ip = trunc(t0);
    const double fp = t0 - ip;
    const long long ticks = (long long)(ip) * 10000000LL + (long long)(fp * 10000000.0);
    return double(ticks) / 10000000.0;
}

// GeoMath.NormalizeLon and GeoMath.Destination (Geo/GeoMath.cs:123-138).
__device__ __forceinline__ double normalize_lon(double lon) {
    lon = fmod(lon + 180.0, 360.0);
    if (lon < 0) lon += 360;
    return lon - 180;
}
__device__ __forceinline__ void destination(double lon, double lat, double az_deg, double dist_km, double& lon2,
                                            double& lat2) {
    const double d = dist_km / kEarthRadiusKm;
    const double p1 = lat * kDeg2Rad, l1 = lon * kDeg2Rad, az = az_deg * kDeg2Rad;
    const double p2 = asin(sin(p1) * cos(d) + cos(p1) * sin(d) * cos(az));
    const double l2 = l1 + atan2(sin(az) * sin(d) * cos(p1), cos(d) - sin(p1) * sin(p2));
    lon2 = normalize_lon(l2 * kRad2Deg);
    lat2 = p2 * kRad2Deg;
}

// EventLocator.Solve (:259-282): Gauss-Jordan with partial pivoting on n <= 4 unknowns; false
// where the reference returns null. The right-hand side is kept as its own column.
__device__ __forceinline__ bool solve_small(const double (&a)[4][4], const double (&b)[4], int n, double (&x)[4]) {
    double m[4][4], rhs[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
#pragma unroll
        for (int j = 0; j < 4; j++) m[i][j] = a[i][j];
        rhs[i] = b[i];
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        if (c < n) {
            int p = c;
            double pv = fabs(m[c][c]);
#pragma unroll
            for (int r = c + 1; r < 4; r++)
                if (r < n && fabs(m[r][c]) > pv) {
                    pv = fabs(m[r][c]);
                    p = r;
                }
            if (pv < 1e-30) return false;
#pragma unroll
            for (int r = c + 1; r < 4; r++)
                if (r == p) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const double tmp = m[c][j];
                        m[c][j] = m[r][j];
                        m[r][j] = tmp;
                    }
                    const double tmp = rhs[c];
                    rhs[c] = rhs[r];
                    rhs[r] = tmp;
                }
#pragma unroll
            for (int r = 0; r < 4; r++) {
                if (r == c || r >= n) continue;
                const double f = m[r][c] / m[c][c];
#pragma unroll
                for (int j = c; j < 4; j++)
                    if (j < n) m[r][j] -= f * m[c][j];
                rhs[r] -= f * rhs[c];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) x[i] = i < n ? rhs[i] / m[i][i] : 0.0;
    return true;
}

// Geiger's Misfit (:173-198) by one warp: lanes evaluate 32 observations at a time, then every lane
// adds their terms in observation order, so all lanes hold the same sums.
__device__ double warp_misfit(const RGrid& g, const ObsD* ob, int n, int npar, double x, double y, double z, double t,
                              bool normal, double (&ata)[4][4], double (&atb)[4], int lane) {
    if (normal) {
#pragma unroll
        for (int a = 0; a < 4; a++) {
            atb[a] = 0;
#pragma unroll
            for (int b = 0; b < 4; b++) ata[a][b] = 0;
        }
    }
    double sum = 0;
    int rows = 0;
    for (int base = 0; base < n; base += 32) {
        const int q = base + lane;
        double res = 0, w = 0, ge = 0, gn = 0, gz = 0;
        bool ok = false;
        if (q < n) {
            const ObsD o = ob[q];
            const double tt = geo::table_time(g, o.tb, x, y, z);
            ok = isfinite(tt);
            if (ok) {
                res = o.sec - t - tt - o.corr;
                w = o.w * o.w;
                if (normal) geo::table_gradient(g, o.tb, x, y, z, ge, gn, gz);
            }
        }
        const unsigned okm = __ballot_sync(kFull, ok);
        const int lim = min(32, n - base);
        for (int l = 0; l < lim; l++) {
            const double rl = __shfl_sync(kFull, res, l);
            const double wl = __shfl_sync(kFull, w, l);
            const double gel = __shfl_sync(kFull, ge, l);
            const double gnl = __shfl_sync(kFull, gn, l);
            const double gzl = __shfl_sync(kFull, gz, l);
            if (!((okm >> l) & 1u)) continue;
            sum += wl * rl * rl;
            rows++;
            if (!normal) continue;
            const double row[4] = {1, gel, gnl, gzl};
#pragma unroll
            for (int a = 0; a < 4; a++) {
                if (a >= npar) continue;
                atb[a] += wl * row[a] * rl;
#pragma unroll
                for (int b = 0; b < 4; b++)
                    if (b < npar) ata[a][b] += wl * row[a] * row[b];
            }
        }
    }
    return rows >= npar ? sum : dinf();
}

// EventLocator.Median (:311-317) of a[0..n) (NaN dropped), sorting a in place. One thread.
__device__ double median_inplace(double* a, int n) {
    int c = 0;
    for (int q = 0; q < n; q++) {
        const double x = a[q];
        if (isnan(x)) continue;
        int p = c++;
        while (p > 0 && a[p - 1] > x) {
            a[p] = a[p - 1];
            p--;
        }
        a[p] = x;
    }
    if (c == 0) return 0;
    return c % 2 == 1 ? a[c / 2] : 0.5 * (a[c / 2 - 1] + a[c / 2]);
}

// Geiger (:166-256) from the grid-search result, then the outlier rule of Locate (:84-90): one warp
// per active event. The event's observations in use are compacted in place when some are rejected.
__global__ void __launch_bounds__(128) geiger_kernel(const RGrid g, const int* __restrict__ active, int n_active,
                                                     const int* __restrict__ off, EvState* __restrict__ st,
                                                     ObsD* __restrict__ olist, int* __restrict__ oidx,
                                                     double* __restrict__ res_buf, double* __restrict__ tmp_buf,
                                                     Params p) {
    const int w = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= n_active) return;
    const int e = active[w];
    EvState s = st[e];
    ObsD* ob = olist + off[e];
    const int n = s.nused;
    const int npar = p.fix_depth ? 3 : 4;
    double lon = s.lon, lat = s.lat, dep = s.dep, t0 = s.t0;
    double ata[4][4], atb[4];
    double lambda = net_max(1e-6, p.damping);
    double chi2 = warp_misfit(g, ob, n, npar, lon, lat, dep, t0, true, ata, atb, lane);
    int it = 0;
    for (; it < p.max_it && isfinite(chi2); it++) {
        bool accepted = false, have = false;
        double step[4] = {0, 0, 0, 0};
        while (lambda < 1e8) {
            double lhs[4][4];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) lhs[a][b] = ata[a][b];
#pragma unroll
            for (int a = 0; a < 4; a++)
                if (a < npar) lhs[a][a] *= 1 + lambda;
            have = solve_small(lhs, atb, npar, step);
            if (!have) break;
            double nlon, nlat;
            destination(lon, lat, atan2(step[1], step[2]) * kRad2Deg, sqrt(step[1] * step[1] + step[2] * step[2]),
                        nlon, nlat);
            const double tlon = net_clamp(geo::unwrap_lon(nlon, g.centre_lon), g.min_lon, g.lon_last);
            const double tlat = net_clamp(nlat, g.min_lat, g.lat_last);
            const double tdep = p.fix_depth ? dep : net_clamp(dep + step[3], g.min_dep, g.dep_last);
            const double tt0 = t0 + step[0];
            const double trial = warp_misfit(g, ob, n, npar, tlon, tlat, tdep, tt0, false, ata, atb, lane);
            if (trial <= chi2) {
                lon = tlon;
                lat = tlat;
                dep = tdep;
                t0 = tt0;
                chi2 = warp_misfit(g, ob, n, npar, lon, lat, dep, t0, true, ata, atb, lane);
                lambda = net_max(1e-6, lambda / 10);
                accepted = true;
                break;
            }
            lambda *= 10;
        }
        if (!accepted || !have) break;
        const double moved = sqrt(step[1] * step[1] + step[2] * step[2] + (npar > 3 ? step[3] * step[3] : 0));
        if (moved < 0.005 && fabs(step[0]) < 0.001) {
            it++;
            break;
        }
    }
    // Covariance from the undamped normal matrix at the solution; Rms over the observations in use.
    warp_misfit(g, ob, n, npar, lon, lat, dep, t0, true, ata, atb, lane);
    double ss = 0;
    for (int base = 0; base < n; base += 32) {
        const int q = base + lane;
        double r = 0;
        if (q < n) r = ob[q].sec - t0 - geo::table_time(g, ob[q].tb, lon, lat, dep) - ob[q].corr;
        const int lim = min(32, n - base);
        for (int l = 0; l < lim; l++) {
            const double rl = __shfl_sync(kFull, r, l);
            ss += rl * rl;
        }
    }
    s.lon = lon;
    s.lat = lat;
    s.dep = dep;
    s.t0 = t0;
    s.rms = sqrt(ss / double(n));
    s.eh = s.emin = s.eaz = s.edep = s.et = dnan();
    double cov[4][4];
    bool inv = true;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        if (c >= npar || !inv) continue;
        double ec[4] = {0, 0, 0, 0}, col[4];
        ec[c] = 1;
        inv = solve_small(ata, ec, npar, col);
#pragma unroll
        for (int r = 0; r < 4; r++) cov[r][c] = col[r];
    }
    if (inv) {
        const double dof = double(max(1, n - npar));
        const double scale = net_max(1, chi2 / dof);
        const double cee = cov[1][1] * scale, cnn = cov[2][2] * scale, cen = cov[1][2] * scale;
        const double tr = 0.5 * (cee + cnn);
        const double det = cee * cnn - cen * cen;
        const double root = sqrt(net_max(0, tr * tr - det));
        s.eh = sqrt(net_max(0, tr + root));
        s.emin = sqrt(net_max(0, tr - root));
        const double theta = 0.5 * atan2(2 * cen, cee - cnn) * kRad2Deg;
        s.eaz = fmod(fmod(90.0 - theta, 180.0) + 180.0, 180.0);
        s.edep = npar > 3 ? sqrt(net_max(0, cov[3][3] * scale)) : 0;
        s.et = sqrt(net_max(0, cov[0][0] * scale));
    }
    s.iterations = it;
    // The outlier rule: residuals at the solution (the origin time as a DateTime holds it), their
    // median and scaled MAD; when a round rejects nothing, or would leave too few phases, the event
    // is done.
    const double tq = tick_seconds(t0);
    double* res = res_buf + off[e];
    double* tmp = tmp_buf + off[e];
    for (int q = lane; q < n; q += 32)
        res[q] = ob[q].sec - tq - geo::table_time(g, ob[q].tb, lon, lat, dep) - ob[q].corr;
    __syncwarp();
    double med = 0, mad = 0;
    if (lane == 0) {
        for (int q = 0; q < n; q++) tmp[q] = res[q];
        med = median_inplace(tmp, n);
        for (int q = 0; q < n; q++) tmp[q] = fabs(res[q] - med);
        mad = 1.4826 * median_inplace(tmp, n);
    }
    med = __shfl_sync(kFull, med, 0);
    mad = __shfl_sync(kFull, mad, 0);
    __syncwarp();
    const double limit = net_max(p.outlier_floor, p.outlier_mads * mad);
    int keep = 0;
    for (int base = 0; base < n; base += 32) {
        const int q = base + lane;
        keep += __popc(__ballot_sync(kFull, q < n && fabs(res[q] - med) <= limit));
    }
    if (keep == n || keep < p.min_phases) {
        s.done = 1;
    } else {
        s.rejected += n - keep;
        // Compact the kept observations in place, in order (a position never passes its source).
        int out = 0;
        for (int base = 0; base < n; base += 32) {
            const int q = base + lane;
            const bool k = q < n && fabs(res[q] - med) <= limit;
            ObsD o{};
            int oi = 0;
            if (q < n) {
                o = ob[q];
                oi = oidx[off[e] + q];
            }
            const unsigned km = __ballot_sync(kFull, k);
            __syncwarp();
            if (k) {
                const int pos = out + __popc(km & ((1u << lane) - 1u));
                ob[pos] = o;
                oidx[off[e] + pos] = oi;
            }
            out += __popc(km);
            __syncwarp();
        }
        s.nused = keep;
    }
    if (lane == 0) st[e] = s;
}

// The residual of every observation of a located event at its solution (EventLocator.cs:92-97).
__global__ void residual_kernel(const RGrid g, int n_obs, const int* __restrict__ oev, const ObsD* __restrict__ oall,
                                const EvState* __restrict__ st, double* __restrict__ out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_obs) return;
    const EvState& s = st[oev[q]];
    if (!s.located) {
        out[q] = dnan();
        return;
    }
    const double tq = tick_seconds(s.t0);
    out[q] = oall[q].sec - tq - geo::table_time(g, oall[q].tb, s.lon, s.lat, s.dep) - oall[q].corr;
}

}  // namespace loc
}  // namespace ts

using namespace ts;
using namespace ts::loc;

namespace {

constexpr int kMaxObs = 1024;  // observations per event (the search kernels' scratch)

int obs_class(int n) { return n <= 32 ? 0 : n <= 128 ? 1 : 2; }

// GeoMath.Azimuth (Geo/GeoMath.cs:98-107) and EventLocator.Gap (Location/EventLocator.cs:320-327).
double azimuth_deg(double lon1, double lat1, double lon2, double lat2) {
    const double p1 = lat1 * kDeg2Rad, p2 = lat2 * kDeg2Rad, dl = (lon2 - lon1) * kDeg2Rad;
    const double y = std::sin(dl) * std::cos(p2);
    const double x = std::cos(p1) * std::sin(p2) - std::sin(p1) * std::cos(p2) * std::cos(dl);
    const double az = std::atan2(y, x) * kRad2Deg;
    return std::fmod(az + 360, 360);
}
double azimuth_gap(const std::vector<double>& az) {
    std::vector<double> a;
    for (double x : az)
        if (std::find(a.begin(), a.end(), x) == a.end()) a.push_back(x);
    std::sort(a.begin(), a.end());
    if (a.size() < 2) return 360;
    double gap = 360 - a.back() + a[0];
    for (size_t i = 1; i < a.size(); i++) gap = std::max(gap, a[i] - a[i - 1]);
    return gap;
}

// Search's box after its clamps (EventLocator.cs:145-153); false when the box is empty.
bool make_task(const host::Grid& g, int e, int i0, int i1, int j0, int j1, int k0, int k1, int stride, int kfix,
               SearchTask& t) {
    i0 = std::max(0, i0); j0 = std::max(0, j0); k0 = std::max(0, k0);
    i1 = std::min(g.nx - 1, i1); j1 = std::min(g.ny - 1, j1); k1 = std::min(g.nz - 1, k1);
    if (kfix >= 0) k0 = k1 = kfix;
    if (i0 > i1 || j0 > j1 || k0 > k1) return false;
    t.event = e;
    t.i0 = i0; t.j0 = j0; t.k0 = k0;
    t.stride = stride;
    t.ci = (i1 - i0) / stride + 1;
    t.cj = (j1 - j0) / stride + 1;
    t.ck = (k1 - k0) / stride + 1;
    t.count = t.ci * t.cj * t.ck;
    t.block0 = 0;
    return true;
}

// E > 0: the warp kernel with E picks per lane; E == 0: the thread kernel.
template <int NMAX, int E>
int run_search(ts_ctx* ctx, const RGrid& rg, std::vector<SearchTask>& tasks, const int* off_d, EvState* st_d,
               const ObsD* olist_d, int fix_depth, std::vector<int>& best, int64_t& candidates) {
    cudaStream_t s = ctx->stream;
    const int per_block = E > 0 ? kBlockCands : kSearchThreads;
    int blocks = 0;
    for (auto& t : tasks) {
        t.block0 = blocks;
        blocks += (t.count + per_block - 1) / per_block;
        candidates += t.count;
    }
    const int nt = int(tasks.size());
    TS_BUF(ctx, tasks_d, SearchTask, "loc.tasks", std::max(1, nt));
    TS_BUF(ctx, part_d, Partial, "loc.partial", std::max(1, blocks));
    TS_BUF(ctx, best_d, int, "loc.best", std::max(1, nt));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(tasks_d, tasks.data(), sizeof(SearchTask) * nt, cudaMemcpyHostToDevice, s));
    if constexpr (E > 0)
        search_warp_kernel<E><<<blocks, kSearchThreads, 0, s>>>(tasks_d, nt, off_d, st_d, olist_d, rg.nx, rg.ny,
                                                                part_d);
    else
        search_kernel<NMAX><<<blocks, kSearchThreads, 0, s>>>(tasks_d, nt, off_d, st_d, olist_d, rg.nx, rg.ny,
                                                              part_d);
    pick_best<NMAX><<<(nt + 127) / 128, 128, 0, s>>>(rg, tasks_d, nt, part_d, off_d, olist_d, st_d, fix_depth,
                                                     per_block, best_d);
    TS_CUDA_TRY(ctx, cudaGetLastError());
    best.resize(nt);
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(best.data(), best_d, sizeof(int) * nt, cudaMemcpyDeviceToHost, s));
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    return TS_OK;
}

int search_classes(ts_ctx* ctx, const RGrid& rg, const std::vector<SearchTask>& tasks, const std::vector<int>& cls,
                   const int* off_d, EvState* st_d, const ObsD* olist_d, int fix_depth, bool dyadic,
                   std::vector<int>& best_of_event, int64_t& candidates) {
    for (int c = 0; c < 3; c++) {
        std::vector<SearchTask> part;
        for (const auto& t : tasks)
            if (cls[t.event] == c) part.push_back(t);
        if (part.empty()) continue;
        std::vector<int> best;
        // Dyadic non-negative weights: one warp per candidate (registers only); otherwise, and above
        // 128 picks, one thread per candidate.
        int rc;
        if (c == 0)
            rc = dyadic ? run_search<32, 1>(ctx, rg, part, off_d, st_d, olist_d, fix_depth, best, candidates)
                        : run_search<32, 0>(ctx, rg, part, off_d, st_d, olist_d, fix_depth, best, candidates);
        else if (c == 1)
            rc = dyadic ? run_search<128, 4>(ctx, rg, part, off_d, st_d, olist_d, fix_depth, best, candidates)
                        : run_search<128, 0>(ctx, rg, part, off_d, st_d, olist_d, fix_depth, best, candidates);
        else
            rc = run_search<kMaxObs, 0>(ctx, rg, part, off_d, st_d, olist_d, fix_depth, best, candidates);
        if (rc) return rc;
        for (size_t k = 0; k < part.size(); k++) best_of_event[part[k].event] = best[k];
    }
    return TS_OK;
}

}  // namespace

extern "C" {

int ts_tables_upload(ts_ctx* ctx, const ts_grid* grid, int32_t n_tables, const float* tables, ts_tables** out) {
    if (!ctx || !out) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = nullptr;
    if (!grid || !tables || n_tables <= 0) return ctx->fail(TS_E_ARG, "bad tables");
    if (const char* bad = host::Grid::validate(*grid)) return ctx->fail(TS_E_ARG, bad);
    if (grid->depth_km) return ctx->fail(TS_E_ARG, "tables need a uniform grid");
    auto* t = new ts_tables();
    t->ctx = ctx;
    t->def = *grid;
    t->n_tables = n_tables;
    t->nodes = int64_t(grid->nx) * grid->ny * grid->nz;
    const size_t bytes = sizeof(float) * size_t(t->nodes) * size_t(n_tables);
    if (cudaMalloc(&t->dev, bytes) != cudaSuccess) {
        cudaGetLastError();
        delete t;
        return ctx->fail(TS_E_NOMEM, "no device memory for the tables");
    }
    if (cudaMemcpy(t->dev, tables, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(t->dev);
        delete t;
        return ctx->fail(TS_E_CUDA, "table upload failed");
    }
    *out = t;
    return TS_OK;
}

int ts_tables_build(ts_ctx* ctx, const ts_grid* grid, const double* slowness, int32_t n_phases, int32_t n_tables,
                    const double* sources, const int32_t* source_phase, int32_t precision, ts_tables** out,
                    ts_eik_stats* stats) {
    if (!ctx || !out) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = nullptr;
    if (stats) *stats = ts_eik_stats{};
    if (!grid || !slowness || !sources || !source_phase || n_tables <= 0 || n_phases <= 0)
        return ctx->fail(TS_E_ARG, "bad tables");
    if (const char* bad = host::Grid::validate(*grid)) return ctx->fail(TS_E_ARG, bad);
    if (grid->depth_km) return ctx->fail(TS_E_ARG, "tables need a uniform grid");
    std::vector<std::pair<int, int>> list(n_tables);
    for (int t = 0; t < n_tables; t++) {
        if (source_phase[t] < 0 || source_phase[t] >= n_phases) return ctx->fail(TS_E_ARG, "phase out of range");
        list[t] = {source_phase[t], t};
    }
    auto* tb = new ts_tables();
    tb->ctx = ctx;
    tb->def = *grid;
    tb->n_tables = n_tables;
    tb->nodes = int64_t(grid->nx) * grid->ny * grid->nz;
    if (cudaMalloc(&tb->dev, sizeof(float) * size_t(tb->nodes) * size_t(n_tables)) != cudaSuccess) {
        cudaGetLastError();
        delete tb;
        return ctx->fail(TS_E_NOMEM, "no device memory for the tables");
    }
    host::Grid g(*grid);
    int rc = precision == TS_PRECISION_F32
                 ? fwd::solve_tables<ts::Pair>(ctx, g, slowness, n_phases, TS_MODE_ENGINE, list, sources, tb->dev, stats)
             : precision == TS_PRECISION_F64
                 ? fwd::solve_tables<double>(ctx, g, slowness, n_phases, TS_MODE_ENGINE, list, sources, tb->dev, stats)
                 : ctx->fail(TS_E_ARG, "precision must be 64 or 32");
    if (rc) {
        cudaFree(tb->dev);
        delete tb;
        return rc;
    }
    *out = tb;
    return TS_OK;
}

int ts_tables_info(ts_tables* t, int32_t* n_tables, int64_t* nodes) {
    if (!t) return TS_E_ARG;
    if (n_tables) *n_tables = t->n_tables;
    if (nodes) *nodes = t->nodes;
    return TS_OK;
}

int ts_tables_copy(ts_tables* t, int32_t first, int32_t count, float* out) {
    if (!t || !out || first < 0 || count < 0 || first + count > t->n_tables) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(t->ctx->mu);
    cudaSetDevice(t->ctx->device);
    const size_t n = size_t(t->nodes);
    TS_CUDA_TRY(t->ctx, cudaMemcpy(out, t->dev + n * first, sizeof(float) * n * count, cudaMemcpyDeviceToHost));
    return TS_OK;
}

void ts_tables_free(ts_tables* t) {
    if (!t) return;
    {
        std::lock_guard<std::recursive_mutex> lk(t->ctx->mu);
        cudaSetDevice(t->ctx->device);
        cudaFree(t->dev);
    }
    delete t;
}

}  // extern "C"

extern "C" int ts_locate(ts_ctx* ctx, ts_tables* tables, const ts_locator_settings* set, int32_t n_events,
                         const double* start, const int32_t* obs_offsets, const int32_t* obs_table,
                         const double* obs_seconds, const double* obs_weight, const double* obs_correction,
                         const double* table_station, ts_location* out, double* residual_out,
                         ts_locate_stats* stats) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (stats) *stats = ts_locate_stats{};
    if (!tables || tables->ctx != ctx) return ctx->fail(TS_E_ARG, "tables belong to another context");
    if (!set || n_events < 0 || (n_events > 0 && (!start || !obs_offsets || !out)))
        return ctx->fail(TS_E_ARG, "bad arguments");
    if (n_events == 0) return TS_OK;
    if (set->coarse_candidates <= 0 || set->min_phases < 0 || set->max_geiger_iterations < 0)
        return ctx->fail(TS_E_ARG, "bad locator settings");
    const int n_obs = obs_offsets[n_events];
    if (obs_offsets[0] != 0 || n_obs < 0) return ctx->fail(TS_E_ARG, "observation offsets must start at 0");
    if (n_obs > 0 && (!obs_table || !obs_seconds || !obs_weight || !obs_correction || !table_station || !residual_out))
        return ctx->fail(TS_E_ARG, "null observation arrays");
    for (int e = 0; e < n_events; e++) {
        const int c = obs_offsets[e + 1] - obs_offsets[e];
        if (c < 0) return ctx->fail(TS_E_ARG, "observation offsets decrease");
        if (c > kMaxObs) return ctx->fail(TS_E_ARG, "an event has more than 1024 observations");
    }
    for (int q = 0; q < n_obs; q++)
        if (obs_table[q] < 0 || obs_table[q] >= tables->n_tables) return ctx->fail(TS_E_ARG, "table index out of range");
    cudaStream_t s = ctx->stream;
    host::Grid g(tables->def);
    const RGrid rg = rays::make_rgrid(g);
    const int fix = set->fix_depth ? 1 : 0;
    EventPair ev;
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    cudaEventRecord(e0, s);
    // Observations (their tables as device pointers), their events, and the per-event state.
    std::vector<ObsD> oall(std::max(1, n_obs));
    std::vector<int> oev(std::max(1, n_obs)), oidx(std::max(1, n_obs));
    for (int e = 0; e < n_events; e++)
        for (int q = obs_offsets[e]; q < obs_offsets[e + 1]; q++) {
            oall[q] = ObsD{tables->dev + size_t(tables->nodes) * size_t(obs_table[q]), obs_seconds[q], obs_weight[q],
                           obs_correction[q]};
            oev[q] = e;
            oidx[q] = q;
        }
    std::vector<EvState> st(n_events);
    std::vector<int> cls(n_events), kfix(n_events, -1), off(obs_offsets, obs_offsets + n_events + 1);
    for (int e = 0; e < n_events; e++) {
        EvState& v = st[e];
        std::memset(&v, 0, sizeof v);
        v.slon = start[3 * e];
        v.slat = start[3 * e + 1];
        v.sdep = start[3 * e + 2];
        v.nused = obs_offsets[e + 1] - obs_offsets[e];
        v.located = v.nused >= set->min_phases && v.nused > 0;
        v.done = !v.located;
        cls[e] = obs_class(v.nused);
        // FixDepth's level (EventLocator.cs:150-153): Math.Round is to even, as nearbyint.
        if (fix) {
            const double fz = (v.sdep - g.min_dep) / g.ddep;
            kfix[e] = std::clamp(int(std::nearbyint(fz)), 0, g.nz - 1);
        }
    }
    const size_t ob = std::max(1, n_obs);
    TS_BUF(ctx, oall_d, ObsD, "loc.oall", ob);
    TS_BUF(ctx, olist_d, ObsD, "loc.olist", ob);
    TS_BUF(ctx, oidx_d, int, "loc.oidx", ob);
    TS_BUF(ctx, oev_d, int, "loc.oev", ob);
    TS_BUF(ctx, res_d, double, "loc.res", ob);
    TS_BUF(ctx, tmp_d, double, "loc.tmp", ob);
    TS_BUF(ctx, off_d, int, "loc.off", n_events + 1);
    TS_BUF(ctx, st_d, EvState, "loc.state", n_events);
    TS_BUF(ctx, act_d, int, "loc.active", n_events);
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(oall_d, oall.data(), sizeof(ObsD) * ob, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(olist_d, oall.data(), sizeof(ObsD) * ob, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(oidx_d, oidx.data(), sizeof(int) * ob, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(oev_d, oev.data(), sizeof(int) * ob, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(off_d, off.data(), sizeof(int) * (n_events + 1), cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(st_d, st.data(), sizeof(EvState) * n_events, cudaMemcpyHostToDevice, s));
    Params prm{set->max_geiger_iterations, set->min_phases, fix, 0, set->damping, set->outlier_mads,
               set->outlier_floor};
    // Weights that are non-negative multiples of 2^-24 below 2^18: any sum of at most 128 of them is
    // exact, whatever the order (the warp search relies on it; otherwise the thread search runs).
    bool dyadic = true;
    for (int q = 0; q < n_obs && dyadic; q++) {
        const double w = obs_weight[q];
        const double sc = std::ldexp(w, 24);
        dyadic = std::isfinite(w) && w >= 0 && w < 262144.0 && sc == std::floor(sc);
    }
    const int stride =
        std::max(1, int(std::ceil(std::cbrt(double(g.count()) / set->coarse_candidates))));  // EventLocator.cs:128
    int64_t candidates = 0;
    int rounds = 0;
    std::vector<int> best(n_events, -1);
    std::vector<char> outside(n_events, 0);
    for (int round = 0; round < 3; round++) {
        std::vector<int> active;
        for (int e = 0; e < n_events; e++)
            if (!st[e].done) active.push_back(e);
        if (active.empty()) break;
        rounds++;
        // The grid search: the whole grid on a stride lattice, then every node around its best
        // (EventLocator.cs:126-132); or every node within 6 of the start (:133-138).
        std::vector<SearchTask> tasks;
        for (int e : active) {
            SearchTask t;
            bool ok;
            if (set->global_search) {
                ok = make_task(g, e, 0, g.nx - 1, 0, g.ny - 1, 0, g.nz - 1, stride, kfix[e], t);
            } else {
                double lon = st[e].slon;
                if (lon < g.centre_lon - 180 || lon > g.centre_lon + 180) lon = host::unwrap_lon(lon, g.centre_lon);
                const int ci = int(std::nearbyint((lon - g.min_lon) / g.dlon));
                const int cj = int(std::nearbyint((st[e].slat - g.min_lat) / g.dlat));
                const int ck = int(std::nearbyint((st[e].sdep - g.min_dep) / g.ddep));
                ok = make_task(g, e, ci - 6, ci + 6, cj - 6, cj + 6, ck - 6, ck + 6, 1, kfix[e], t);
            }
            if (ok) tasks.push_back(t);
            else outside[e] = 1;
        }
        int rc = search_classes(ctx, rg, tasks, cls, off_d, st_d, olist_d, fix, dyadic, best, candidates);
        if (rc) return rc;
        if (set->global_search) {
            std::vector<SearchTask> fine;
            for (const auto& t0 : tasks) {
                const int b = best[t0.event];
                const int bi = b % g.nx, bj = (b / g.nx) % g.ny, bk = b / (g.nx * g.ny);
                SearchTask t;
                if (make_task(g, t0.event, bi - 2 * stride, bi + 2 * stride, bj - 2 * stride, bj + 2 * stride,
                              bk - 2 * stride, bk + 2 * stride, 1, kfix[t0.event], t))
                    fine.push_back(t);
            }
            rc = search_classes(ctx, rg, fine, cls, off_d, st_d, olist_d, fix, dyadic, best, candidates);
            if (rc) return rc;
        }
        // Geiger and the outlier rule for the events whose search ran.
        std::vector<int> run;
        for (int e : active)
            if (!outside[e]) run.push_back(e);
        if (!run.empty()) {
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(act_d, run.data(), sizeof(int) * run.size(), cudaMemcpyHostToDevice, s));
            const int warps = int(run.size());
            geiger_kernel<<<(warps + 3) / 4, 128, 0, s>>>(rg, act_d, warps, off_d, st_d, olist_d, oidx_d, res_d,
                                                          tmp_d, prm);
            TS_CUDA_TRY(ctx, cudaGetLastError());
        }
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(st.data(), st_d, sizeof(EvState) * n_events, cudaMemcpyDeviceToHost, s));
        TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        bool changed = false;
        for (int e : active)
            if (outside[e]) {
                st[e].done = 1;
                st[e].located = 0;
                changed = true;
            }
        if (changed)
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(st_d, st.data(), sizeof(EvState) * n_events, cudaMemcpyHostToDevice, s));
    }
    if (n_obs > 0) {
        residual_kernel<<<(n_obs + 255) / 256, 256, 0, s>>>(rg, n_obs, oev_d, oall_d, st_d, res_d);
        TS_CUDA_TRY(ctx, cudaGetLastError());
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(residual_out, res_d, sizeof(double) * n_obs, cudaMemcpyDeviceToHost, s));
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(oidx.data(), oidx_d, sizeof(int) * n_obs, cudaMemcpyDeviceToHost, s));
    }
    cudaEventRecord(e1, s);
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double nan = std::nan("");
    for (int e = 0; e < n_events; e++) {
        const EvState& v = st[e];
        ts_location& r = out[e];
        if (!v.located) {
            // Too few phases: LocationResult(start, count, 0, 0, ...) (EventLocator.cs:74-75). A local
            // search box outside the grid: the reference reads past its table and Relocation.Absolute
            // reports the exception with nothing used (Relocation.cs:84-86).
            r = ts_location{0, v.slon, v.slat, v.sdep, nan, nan, nan, nan, nan, nan, nan,
                            outside[e] ? 0 : obs_offsets[e + 1] - obs_offsets[e], 0, 0, outside[e] ? 2 : 1};
            continue;
        }
        std::vector<double> az;
        for (int p = 0; p < v.nused; p++) {
            const int t = obs_table[oidx[obs_offsets[e] + p]];
            az.push_back(azimuth_deg(v.lon, v.lat, table_station[2 * t], table_station[2 * t + 1]));
        }
        r = ts_location{v.t0, v.lon, v.lat, v.dep, v.rms, v.eh, v.emin, v.eaz, v.edep, v.et, azimuth_gap(az),
                        v.nused, v.rejected, v.iterations, 0};
    }
    if (stats) {
        stats->device_ms = ms;
        stats->candidates = candidates;
        stats->rounds = rounds;
    }
    return TS_OK;
}
