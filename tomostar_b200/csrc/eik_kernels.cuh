// Eikonal sweeping kernels: the plain per-plane kernel (the reference's launch scheme) and the
// tiled engine (one cooperative persistent launch over many fields and grids).
//
// Why the tiled engine gives the reference's result to the bit. A sweep of ordering `dir` visits
// the nodes by diagonal planes i'+j'+k' = p (mirrored coordinates), Gauss-Seidel in place
// (SphericalEikonal.cs:297-321). A node's update reads its neighbours one and two steps away on
// each axis; those on smaller p are already updated in this sweep, those on larger p are not yet.
// Any visiting order in which every node comes after its axis neighbours of smaller p produces
// exactly the same values. The engine cuts the grid into BX×BY×BZ tiles and visits them by tile
// diagonals a'+b'+c' = q (all tiles of one diagonal at once: no two are face neighbours, and the
// stencil only reaches face neighbours), and inside a tile by node planes. Every axis neighbour of
// smaller p lies in the same tile or in a tile of smaller q, so the order is one of those orders.
// Skipping a tile none of whose nodes has an input that moved since its last evaluation skips
// only updates that would return the value already held, as the reference's dirty flags do
// (EikonalOpenCl.cs:529-532, 608-622); the field is unchanged by it.
#pragma once

#include "eik_update.cuh"

namespace ts {
namespace eik {

// ---- plain path: one launch per diagonal plane of one field (EikonalOpenCl.cs:232-268, 506-623) --

template <typename Real, bool VARZ>
__global__ void plain_sweep_kernel(Real* __restrict__ T, const Real* __restrict__ slow, const uint8_t* __restrict__ fixed,
                                   uint8_t* __restrict__ dirty, const Real* __restrict__ wx,
                                   const Real* __restrict__ wy, Real wz1, Real wz2, const Real* __restrict__ zc, int nx, int ny,
                                   int nz, int second, int* changed, int dir, int p, Real tol,
                                   unsigned long long* updates) {
    int i0 = max(0, p - (ny - 1) - (nz - 1));
    int iw = min(nx - 1, p) - i0 + 1;
    int k0 = max(0, p - (nx - 1) - (ny - 1));
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    bool did = false;
    if (a < iw) {
        int ip = i0 + a, kp = k0 + int(blockIdx.y), jp = p - ip - kp;
        if (jp >= 0 && jp < ny) {
            int i = (dir & 1) ? nx - 1 - ip : ip;
            int j = (dir & 2) ? ny - 1 - jp : jp;
            int k = (dir & 4) ? nz - 1 - kp : kp;
            int nxy = nx * ny;
            int node = (k * ny + j) * nx + i;
            if (!fixed[node] && dirty[node]) {
                dirty[node] = 0;
                did = true;
                const Real inf = real_inf<Real>();
                Real cur = T[node];
                Real cand = Update<Real, VARZ>::eval(
                    slow[node], i > 0 ? T[node - 1] : inf, i + 1 < nx ? T[node + 1] : inf,
                    i > 1 ? T[node - 2] : inf, i + 2 < nx ? T[node + 2] : inf, j > 0 ? T[node - nx] : inf,
                    j + 1 < ny ? T[node + nx] : inf, j > 1 ? T[node - 2 * nx] : inf,
                    j + 2 < ny ? T[node + 2 * nx] : inf, k > 0 ? T[node - nxy] : inf,
                    k + 1 < nz ? T[node + nxy] : inf, k > 1 ? T[node - 2 * nxy] : inf,
                    k + 2 < nz ? T[node + 2 * nxy] : inf, wx[2 * (k * ny + j)], wx[2 * (k * ny + j) + 1],
                    wy[2 * k], wy[2 * k + 1], wz1, wz2, VARZ ? zc + kZCoef * k : nullptr, second != 0);
                if (cand < cur) {
                    T[node] = cand;
                    if (counts_as_change<Real>(cur, cand, tol)) atomicOr(changed, 1);
                    // Wake the nodes that read this one (EikonalOpenCl.cs:608-622).
                    if (i > 0) dirty[node - 1] = 1;
                    if (i > 1) dirty[node - 2] = 1;
                    if (i + 1 < nx) dirty[node + 1] = 1;
                    if (i + 2 < nx) dirty[node + 2] = 1;
                    if (j > 0) dirty[node - nx] = 1;
                    if (j > 1) dirty[node - 2 * nx] = 1;
                    if (j + 1 < ny) dirty[node + nx] = 1;
                    if (j + 2 < ny) dirty[node + 2 * nx] = 1;
                    if (k > 0) dirty[node - nxy] = 1;
                    if (k > 1) dirty[node - 2 * nxy] = 1;
                    if (k + 1 < nz) dirty[node + nxy] = 1;
                    if (k + 2 < nz) dirty[node + 2 * nxy] = 1;
                }
            }
        }
    }
    unsigned m = __ballot_sync(0xffffffffu, did);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(updates, (unsigned long long)__popc(m));
}

template <typename Real>
__global__ void fill_kernel(Real* __restrict__ p, Real v, int64_t n) {
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n; q += int64_t(gridDim.x) * blockDim.x) p[q] = v;
}

__global__ void fill_u8_kernel(uint8_t* __restrict__ p, uint8_t v, int64_t n);

// Writes seed times (already min-merged per field) and, for the plain path, the fixed mask.
template <typename Real>
__global__ void seed_kernel(Real* __restrict__ T, uint8_t* __restrict__ fixed, const int64_t* __restrict__ at,
                            const double* __restrict__ t, int count) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    T[at[q]] = Real(t[q]);
    if (fixed) fixed[at[q]] = 1;
}

// ---- tiled engine ---------------------------------------------------------------------------------

enum FieldStatus : int { kRunning = 0, kSettled = 1, kUnsettled = 2 };

// One grid shape and its metric (shared by every field solved on it).
struct GridDesc {
    int nx, ny, nz;
    int tx, ty, tz;            // tile counts
    int ndiag;                 // tile diagonals: tx + ty + tz - 2
    int varz;                  // variable vertical spacing (extension)
    const int* diag_off;       // [ndiag + 1] offsets into diag_tiles
    const uint32_t* diag_tiles;// canonical tile coords (a | b << 10 | c << 20), ordered by a + b + c
    const void* wx;            // Real[2 * nz * ny]: longitude-axis weights (w1, w2) per (k, j)
    const void* wy;            // Real[2 * nz]: latitude-axis weights per k
    const void* zc;            // Real[kZCoef * nz] when varz
    double wz1, wz2;           // depth-axis weights of a uniform grid
    int pitch;                 // elements per padded field row (see FieldDesc::T)
    int pad;
};

// The engine's field layout: every (k, j) row is padded to `pitch` elements, node (i, j, k) at
// (k·ny + j)·pitch + HX + i with HX = 16 / sizeof(Real); the pads hold +inf and are never written.
// A tile's row segment with its two-node x halo is then one 16-byte-aligned run of whole chunks.
template <typename Real>
struct Layout {
    static constexpr int HX = 16 / int(sizeof(Real));
    TS_HDINL static int pitch(int tiles_x, int bx) { return HX + tiles_x * bx + HX; }
};

template <typename Real>
struct FieldDesc {
    Real* T;              // the field, padded rows (Layout)
    const Real* s;        // its slowness
    uint8_t* dirty;       // one flag per tile
    int grid;             // GridDesc index
    int seed_begin;       // its seed tiles: seed_tile[seed_begin .. seed_begin + seed_count), by tile id
    int seed_count;
    int cap;              // round cap per phase
};

struct FieldState {
    int phase, round, status, changed;
    int enter1, rounds0, rounds1, pad;
};

struct Control {
    unsigned int bar_count;
    unsigned int bar_gen;
    int abort;
    int error;
    int running;
    int cancelled;
    int epochs;
    int pad;
    unsigned long long updates;
    unsigned long long visits;
};

struct Plan {
    int ngroups;
    int maxdiag;
    const int* group_grid;   // [ngroups]
    const int* group_first;  // [ngroups] first entry of the group in field_list
    const int* field_list;   // fields ordered by group
    const int* pre;          // [maxdiag][ngroups + 1] item prefix of each diagonal step
};

template <typename Real>
struct Args {
    const GridDesc* grids;
    const FieldDesc<Real>* fields;
    FieldState* state;
    const int* seed_tile;        // tile id of each seed tile
    const uint32_t* seed_mask;   // kMaskWords words per seed tile: the fixed nodes
    const uint16_t* plane_tab;   // canonical tile nodes ordered by plane
    const int* plane_off;        // [nplanes + 1]
    Control* ctl;
    const volatile int* cancel;  // host-mapped cancel flag
    Plan plan;
    int n_active;                // entries of plan.field_list
    int max_rounds_per_launch;   // rounds this launch may run (<= 0: until every field is done)
    long long barrier_timeout_ns;
    Real tol;
};

TS_DEVINL unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier of a cooperative launch with a bounded wait: a block that waits longer than
// the limit raises abort and the error, and every block leaves at its next barrier. Returns
// false when the launch is aborting.
TS_DEVINL bool grid_barrier(Control* c, unsigned nblocks, long long timeout_ns) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned* gen = &c->bar_gen;
        unsigned g = *gen;
        __threadfence();
        unsigned arrived = atomicAdd(&c->bar_count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&c->bar_count, 0u);
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        } else {
            unsigned long long t0 = global_ns();
            while (*gen == g) {
                if (*(volatile int*)&c->abort) { ok = 0; break; }
                if ((long long)(global_ns() - t0) > timeout_ns) {
                    atomicCAS(&c->error, 0, TS_E_TIMEOUT);
                    atomicExch(&c->abort, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (*(volatile int*)&c->abort) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

template <typename Real, int BX_, int BY_, int BZ_>
struct Shape {
    static constexpr int BX = BX_, BY = BY_, BZ = BZ_;
    static constexpr int N = BX * BY * BZ;
    static constexpr int HX = Layout<Real>::HX;
    static constexpr int CX = BX + 2 * HX, CY = BY + 4, CZ = BZ + 4;
    static constexpr int CUBE = CX * CY * CZ;
    static constexpr int NCH = CX / HX;  // 16-byte chunks per cube row
    static constexpr int NPLANES = BX + BY + BZ - 2;
    static constexpr int MW = (N + 31) / 32;
    static_assert(BX % HX == 0, "tile rows must be whole 16-byte chunks");
    TS_HDINL static int cidx(int i, int j, int k) { return ((k + 2) * CY + (j + 2)) * CX + (i + HX); }
};

// Shared memory of one warp's tile: the node cube with a two-node halo on each face, the tile's
// slowness, its axis weights and its fixed-node mask.
template <class S>
constexpr int warp_reals() {
    return S::CUBE + S::N + 2 * S::BY * S::BZ + 2 * S::BZ + kZCoef * S::BZ;
}

template <typename Real, class S>
struct WarpSmem {
    static constexpr int kBytes = ((warp_reals<S>() * int(sizeof(Real)) + S::MW * 4) + 15) / 16 * 16;
};

template <typename Real, class S>
constexpr int engine_smem_bytes(int warps) {
    return warps * WarpSmem<Real, S>::kBytes + ((S::N * 2 + 15) / 16 * 16) + (S::NPLANES + 1) * 4;
}

// Processes one tile of one field for sweep ordering `dir`. Returns the node evaluations made.
template <typename Real, class S, bool VARZ>
TS_DEVINL int process_tile(const Args<Real>& a, const GridDesc& g, const FieldDesc<Real>& fd, int f, int tx, int ty,
                           int tz, int dir, bool second, Real* cube, Real* ss, Real* mwx, Real* mwy, Real* mzc,
                           uint32_t* mask, const uint16_t* ptab, const int* poff, int lane) {
    const Real inf = real_inf<Real>();
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t nxy = int64_t(nx) * ny;
    const int x0 = tx * S::BX, y0 = ty * S::BY, z0 = tz * S::BZ;
    const int tid = (tz * g.ty + ty) * g.tx + tx;
    Real* __restrict__ T = fd.T;
    const Real* __restrict__ slow = fd.s;
    if (lane == 0) __stcg(&fd.dirty[tid], (uint8_t)0);

    // Axis weights of the tile's rows.
    const Real* wx = static_cast<const Real*>(g.wx);
    const Real* wy = static_cast<const Real*>(g.wy);
    for (int q = lane; q < 2 * S::BY * S::BZ; q += 32) {
        int r = q >> 1, j = y0 + r % S::BY, k = z0 + r / S::BY;
        mwx[q] = (j < ny && k < nz) ? __ldg(&wx[2 * (int64_t(k) * ny + j) + (q & 1)]) : Real(1);
    }
    for (int q = lane; q < 2 * S::BZ; q += 32) mwy[q] = (z0 + (q >> 1) < nz) ? __ldg(&wy[2 * z0 + q]) : Real(1);
    if (VARZ) {
        const Real* zc = static_cast<const Real*>(g.zc);
        for (int q = lane; q < kZCoef * S::BZ; q += 32) {
            int k = z0 + q / kZCoef;
            mzc[q] = k < nz ? __ldg(&zc[int64_t(k) * kZCoef + q % kZCoef]) : Real(1);
        }
    }
    // The cube: every row segment the stencil reads (the interior rows with their x halo, and the
    // y and z halo rows; the corner rows are never read), as asynchronous 16-byte copies, +inf for
    // rows off the grid. The pads of a field row hold +inf, so x needs no check.
    const int pitch = g.pitch;
    for (int q = lane; q < S::CY * S::CZ * S::NCH; q += 32) {
        int row = q / S::NCH, ch = q - row * S::NCH;
        int jj = row % S::CY - 2, kk = row / S::CY - 2;
        bool yin = jj >= 0 && jj < S::BY, zin = kk >= 0 && kk < S::BZ;
        if (!yin && !zin) continue;
        Real* dst = cube + row * S::CX + ch * S::HX;
        int gy = y0 + jj, gz = z0 + kk;
        if (gy >= 0 && gy < ny && gz >= 0 && gz < nz) {
            cp_async16_cg(dst, T + (int64_t(gz) * ny + gy) * pitch + x0 + ch * S::HX);
        } else {
#pragma unroll
            for (int e = 0; e < S::HX; e++) dst[e] = inf;
        }
    }
    // Slowness of the tile's nodes (read-only, dense grid order).
    for (int q = lane; q < S::N; q += 32) {
        int i = q % S::BX, j = (q / S::BX) % S::BY, k = q / (S::BX * S::BY);
        int gx = x0 + i, gy = y0 + j, gz = z0 + k;
        if (gx < nx && gy < ny && gz < nz) cp_async_ro(&ss[q], &slow[gz * nxy + int64_t(gy) * nx + gx]);
        else ss[q] = Real(0);
    }
    // Fixed (seed) nodes of this tile, if any: binary search of the field's seed tiles.
    {
        int lo = 0, hi = fd.seed_count;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (__ldg(&a.seed_tile[fd.seed_begin + mid]) < tid) lo = mid + 1;
            else hi = mid;
        }
        bool has = lo < fd.seed_count && __ldg(&a.seed_tile[fd.seed_begin + lo]) == tid;
        for (int q = lane; q < S::MW; q += 32)
            mask[q] = has ? __ldg(&a.seed_mask[int64_t(fd.seed_begin + lo) * S::MW + q]) : 0u;
    }
    cp_async_wait_all();
    __syncwarp();

    // Node planes of the tile in the mirrored order of `dir`.
    const Real tol = a.tol;
    bool any = false, big = false;
    unsigned faces = 0;
    int evals = 0;
    for (int p = 0; p < S::NPLANES; p++) {
        int e1 = poff[p + 1];
        for (int e = poff[p] + lane; e < e1; e += 32) {
            unsigned pk = ptab[e];
            int ip = pk & 31, jp = (pk >> 5) & 31, kp = pk >> 10;
            int i = (dir & 1) ? S::BX - 1 - ip : ip;
            int j = (dir & 2) ? S::BY - 1 - jp : jp;
            int k = (dir & 4) ? S::BZ - 1 - kp : kp;
            if (x0 + i >= nx || y0 + j >= ny || z0 + k >= nz) continue;
            int L = (k * S::BY + j) * S::BX + i;
            if ((mask[L >> 5] >> (L & 31)) & 1u) continue;
            evals++;
            int c = S::cidx(i, j, k);
            Real cur = cube[c];
            Real cand = Update<Real, VARZ>::eval(
                ss[L], cube[c - 1], cube[c + 1], cube[c - 2], cube[c + 2], cube[c - S::CX], cube[c + S::CX],
                cube[c - 2 * S::CX], cube[c + 2 * S::CX], cube[c - S::CX * S::CY], cube[c + S::CX * S::CY],
                cube[c - 2 * S::CX * S::CY], cube[c + 2 * S::CX * S::CY], mwx[2 * (k * S::BY + j)],
                mwx[2 * (k * S::BY + j) + 1], mwy[2 * k], mwy[2 * k + 1], Real(g.wz1), Real(g.wz2),
                VARZ ? mzc + kZCoef * k : nullptr, second);
            if (cand < cur) {
                cube[c] = cand;
                any = true;
                if (counts_as_change<Real>(cur, cand, tol)) big = true;
                faces |= (i < 2 ? 1u : 0u) | (i >= S::BX - 2 ? 2u : 0u) | (j < 2 ? 4u : 0u) |
                         (j >= S::BY - 2 ? 8u : 0u) | (k < 2 ? 16u : 0u) | (k >= S::BZ - 2 ? 32u : 0u);
            }
        }
        __syncwarp();
    }
    bool any_w = __any_sync(0xffffffffu, any);
    if (any_w) {
        bool big_w = __any_sync(0xffffffffu, big);
        unsigned faces_w = __reduce_or_sync(0xffffffffu, faces);
        for (int q = lane; q < S::N; q += 32) {
            int i = q % S::BX, j = (q / S::BX) % S::BY, k = q / (S::BX * S::BY);
            int gx = x0 + i, gy = y0 + j, gz = z0 + k;
            if (gx < nx && gy < ny && gz < nz) st_cg(&T[(int64_t(gz) * ny + gy) * pitch + S::HX + gx], cube[S::cidx(i, j, k)]);
        }
        // A node of this tile may read a node that changed after it was evaluated: visit the tile
        // again next sweep. Neighbour tiles within two nodes of a changed node are woken too.
        if (lane == 0) __stcg(&fd.dirty[tid], (uint8_t)1);
        if (lane == 1 && (faces_w & 1u) && tx > 0) __stcg(&fd.dirty[tid - 1], (uint8_t)1);
        if (lane == 2 && (faces_w & 2u) && tx + 1 < g.tx) __stcg(&fd.dirty[tid + 1], (uint8_t)1);
        if (lane == 3 && (faces_w & 4u) && ty > 0) __stcg(&fd.dirty[tid - g.tx], (uint8_t)1);
        if (lane == 4 && (faces_w & 8u) && ty + 1 < g.ty) __stcg(&fd.dirty[tid + g.tx], (uint8_t)1);
        if (lane == 5 && (faces_w & 16u) && tz > 0) __stcg(&fd.dirty[tid - g.tx * g.ty], (uint8_t)1);
        if (lane == 6 && (faces_w & 32u) && tz + 1 < g.tz) __stcg(&fd.dirty[tid + g.tx * g.ty], (uint8_t)1);
        if (lane == 7 && big_w) atomicExch(&a.state[f].changed, 1);
    }
    __syncwarp();
    return evals;
}

template <typename Real, int BX, int BY, int BZ, int WARPS, bool VARZ_ANY>
__global__ void __launch_bounds__(WARPS * 32) engine_kernel(Args<Real> a) {
    using S = Shape<Real, BX, BY, BZ>;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int kWarpBytes = WarpSmem<Real, S>::kBytes;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* mine = smem + warp * kWarpBytes;
    Real* cube = reinterpret_cast<Real*>(mine);
    Real* ss = cube + S::CUBE;
    Real* mwx = ss + S::N;
    Real* mwy = mwx + 2 * S::BY * S::BZ;
    Real* mzc = mwy + 2 * S::BZ;
    uint32_t* mask = reinterpret_cast<uint32_t*>(mzc + kZCoef * S::BZ);
    uint16_t* ptab = reinterpret_cast<uint16_t*>(smem + WARPS * kWarpBytes);
    int* poff = reinterpret_cast<int*>(smem + WARPS * kWarpBytes + (S::N * 2 + 15) / 16 * 16);
    for (int q = threadIdx.x; q < S::N; q += blockDim.x) ptab[q] = a.plane_tab[q];
    for (int q = threadIdx.x; q <= S::NPLANES; q += blockDim.x) poff[q] = a.plane_off[q];
    __syncthreads();

    const unsigned nblocks = gridDim.x;
    const int gwarp = blockIdx.x * WARPS + warp;
    const int nwarps = nblocks * WARPS;
    const int G = a.plan.ngroups;
    unsigned long long my_updates = 0, my_visits = 0;
    int rounds_this_launch = 0;

    for (;;) {
        for (int dir = 0; dir < 8; dir++) {
            for (int q = 0; q < a.plan.maxdiag; q++) {
                const int* pre = a.plan.pre + int64_t(q) * (G + 1);
                const int total = __ldg(&pre[G]);
                // Items are dealt round-robin to the warps (item = gwarp + j·nwarps), so a small step
                // still spreads over the whole GPU. Each lane decodes one of the warp's next 32
                // items; the warp then processes the dirty ones in turn.
                for (int64_t j0 = 0; gwarp + j0 * nwarps < total; j0 += 32) {
                    int64_t item64 = gwarp + (j0 + lane) * nwarps;
                    int item = item64 < total ? int(item64) : total;
                    int f = -1, tx = 0, ty = 0, tz = 0;
                    if (item < total) {
                        int lo = 0, hi = G;  // first g with pre[g] > item, minus one
                        while (lo < hi) {
                            int mid = (lo + hi) >> 1;
                            if (__ldg(&pre[mid + 1]) <= item) lo = mid + 1;
                            else hi = mid;
                        }
                        const int grp = lo;
                        const GridDesc& g = a.grids[__ldg(&a.plan.group_grid[grp])];
                        int d0 = __ldg(&g.diag_off[q]);
                        int cnt = __ldg(&g.diag_off[q + 1]) - d0;
                        int li = item - __ldg(&pre[grp]);
                        int fi = li / cnt, ti = li - fi * cnt;
                        int fld = __ldg(&a.plan.field_list[__ldg(&a.plan.group_first[grp]) + fi]);
                        uint32_t pk = __ldg(&g.diag_tiles[d0 + ti]);
                        int ca = pk & 1023, cb = (pk >> 10) & 1023, cc = pk >> 20;
                        tx = (dir & 1) ? g.tx - 1 - ca : ca;
                        ty = (dir & 2) ? g.ty - 1 - cb : cb;
                        tz = (dir & 4) ? g.tz - 1 - cc : cc;
                        const FieldState* st = &a.state[fld];
                        if (*(volatile const int*)&st->status == kRunning) {
                            const FieldDesc<Real>& fd = a.fields[fld];
                            if (__ldcg(&fd.dirty[(tz * g.ty + ty) * g.tx + tx])) f = fld;
                        }
                    }
                    unsigned m = __ballot_sync(0xffffffffu, f >= 0);
                    while (m) {
                        int src = __ffs(m) - 1;
                        m &= m - 1;
                        int ff = __shfl_sync(0xffffffffu, f, src);
                        int sx = __shfl_sync(0xffffffffu, tx, src);
                        int sy = __shfl_sync(0xffffffffu, ty, src);
                        int sz = __shfl_sync(0xffffffffu, tz, src);
                        const FieldDesc<Real>& fd = a.fields[ff];
                        const GridDesc& g = a.grids[fd.grid];
                        bool second = *(volatile const int*)&a.state[ff].phase == 1;
                        int ev;
                        if (VARZ_ANY && g.varz)
                            ev = process_tile<Real, S, true>(a, g, fd, ff, sx, sy, sz, dir, second, cube, ss, mwx,
                                                             mwy, mzc, mask, ptab, poff, lane);
                        else
                            ev = process_tile<Real, S, false>(a, g, fd, ff, sx, sy, sz, dir, second, cube, ss, mwx,
                                                              mwy, mzc, mask, ptab, poff, lane);
                        my_updates += ev;
                        my_visits += 1;
                    }
                }
                if (!grid_barrier(a.ctl, nblocks, a.barrier_timeout_ns)) goto done;
            }
        }
        // Round end: each running field settles, moves to phase 1, or is refused at the cap
        // (SphericalEikonal.cs:297-323; EikonalOpenCl.cs:241-269).
        {
            int t = blockIdx.x * blockDim.x + threadIdx.x;
            if (t == 0) a.ctl->cancelled = (a.cancel && *a.cancel) ? 1 : 0;
            for (int e = t; e < a.n_active; e += nblocks * blockDim.x) {
                int fld = a.plan.field_list[e];
                volatile FieldState* st = &a.state[fld];
                if (st->status != kRunning) continue;
                int cap = a.fields[fld].cap;
                if (!st->changed) {
                    if (st->phase == 0) {
                        st->rounds0 = st->round + 1;
                        st->phase = 1;
                        st->round = 0;
                        st->enter1 = 1;
                    } else {
                        st->rounds1 = st->round + 1;
                        st->status = kSettled;
                        atomicSub(&a.ctl->running, 1);
                    }
                } else {
                    st->round += 1;
                    if (st->round >= cap) {
                        if (st->phase == 0) st->rounds0 = st->round;
                        else st->rounds1 = st->round;
                        st->status = kUnsettled;
                        atomicSub(&a.ctl->running, 1);
                    }
                }
                st->changed = 0;
            }
        }
        if (!grid_barrier(a.ctl, nblocks, a.barrier_timeout_ns)) goto done;
        // Phase 1 starts with every node due for an update (EikonalOpenCl.cs:235-239).
        for (int e = blockIdx.x; e < a.n_active; e += nblocks) {
            int fld = a.plan.field_list[e];
            if (!*(volatile int*)&a.state[fld].enter1) continue;
            const FieldDesc<Real>& fd = a.fields[fld];
            const GridDesc& g = a.grids[fd.grid];
            int nt = g.tx * g.ty * g.tz;
            for (int q = threadIdx.x; q < nt; q += blockDim.x) __stcg(&fd.dirty[q], (uint8_t)1);
            __syncthreads();
            if (threadIdx.x == 0) a.state[fld].enter1 = 0;
        }
        rounds_this_launch++;
        if (!grid_barrier(a.ctl, nblocks, a.barrier_timeout_ns)) goto done;
        if (*(volatile int*)&a.ctl->running <= 0) break;
        if (*(volatile int*)&a.ctl->cancelled) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(&a.ctl->error, 0, TS_E_CANCELLED);
            break;
        }
        if (a.max_rounds_per_launch > 0 && rounds_this_launch >= a.max_rounds_per_launch) break;
    }
done:
    for (int o = 16; o > 0; o >>= 1) my_updates += __shfl_down_sync(0xffffffffu, my_updates, o);
    if (lane == 0) {
        atomicAdd(&a.ctl->updates, my_updates);
        atomicAdd(&a.ctl->visits, my_visits);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.ctl->epochs, rounds_this_launch);
}

}  // namespace eik
}  // namespace ts
