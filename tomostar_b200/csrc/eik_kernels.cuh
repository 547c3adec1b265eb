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

struct FieldState {
    int phase, round, status, changed;
    int enter1, rounds0, rounds1, pad;
    // Flow scheduler: the sweep ordering and diagonal in progress, its tiles still outstanding, and
    // the rounds run in the current launch.
    int dir, q, pending, launch_rounds;
    int pad2[4];
};

template <typename Real>
struct FieldDesc {
    Real* T;              // the field, padded rows (Layout)
    const Real* s;        // its slowness
    uint8_t* dirty;       // one flag per tile: some node of the tile is due for an update
    uint32_t* dmask;      // per tile, one bit per node (MW words): the node is due for an update
    int grid;             // GridDesc index
    int seed_begin;       // its seed tiles: seed_tile[seed_begin .. seed_begin + seed_count), by tile id
    int seed_count;
    int cap;              // round cap per phase
    int seed_tile_lo, seed_tile_hi;  // smallest and largest seed tile id (no search outside)
    FieldState* state;               // the field's solve state; lives with the field between launches
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
    int produced[2];   // due tiles listed in the step's worklist (by step parity)
    int consumed[2];   // worklist entries taken
    // Flow scheduler: the tile queue's tickets (consumers take from head, producers reserve at tail)
    // and the end of the launch (every field stopped).
    unsigned long long q_head, q_tail;
    unsigned long long t_start;  // globaltimer at the launch's start (first warp to arrive)
    int done;
    int pad3[3];
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
    const int* seed_tile;        // tile id of each seed tile
    const uint32_t* seed_mask;   // kMaskWords words per seed tile: the fixed nodes
    const uint16_t* plane_tab;   // canonical tile nodes ordered by plane
    const int* plane_off;        // [nplanes + 1]
    const uint32_t* wake_mask;   // [12][MW] destination masks of the 12 stencil offsets (see wake)
    Control* ctl;
    const volatile int* cancel;  // host-mapped cancel flag
    Plan plan;
    int n_active;                // entries of plan.field_list
    unsigned long long* worklist;  // 2 x worklist_cap due tiles: field << 32 | tx | ty << 10 | tz << 20
    int worklist_cap;
    int max_rounds_per_launch;   // rounds this launch may run (<= 0: until every field is done)
    long long epoch_budget_ns;   // flow scheduler: after this long, each field pauses at its next round end
    long long barrier_timeout_ns;
    // Flow scheduler queue (a bounded multi-producer multi-consumer ring): items[slot] =
    // field << 32 | tx | ty << 10 | tz << 20. seq[slot] starts at slot; the producer of ticket t waits
    // for seq == t, writes, and sets t + 1; its consumer waits for t + 1, reads, and sets t + capacity.
    unsigned long long* q_items;
    unsigned long long* q_seq;
    unsigned long long q_mask;
    Real tol;
    Real wake_rel;               // a drop wakes the neighbours when it exceeds wake_rel × the new time
    int causal;                  // a drop to t wakes only the neighbours holding more than t
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

// Per warp also four node bitsets of MW words: fixed (seed) nodes, due nodes, nodes changed in the
// current plane, nodes changed in this visit.
template <typename Real, class S>
struct WarpSmem {
    static constexpr int kBytes = ((warp_reals<S>() * int(sizeof(Real)) + 4 * S::MW * 4) + 15) / 16 * 16;
};

// The 12 stencil offsets in a tile's linear node index, in the order of the wake masks.
template <class S>
TS_HDINL int stencil_offset(int d) {
    const int step[3] = {1, S::BX, S::BX * S::BY};
    int axis = d >> 2, r = d & 3;  // r: +1, -1, +2, -2
    int m = (r & 2) ? 2 : 1;
    return ((r & 1) ? -m : m) * step[axis];
}

template <typename Real, class S>
constexpr int engine_smem_bytes(int warps) {
    return warps * WarpSmem<Real, S>::kBytes + ((S::N * 2 + 15) / 16 * 16) + ((S::NPLANES + 1) * 4 + 15) / 16 * 16 +
           12 * S::MW * 4;
}

// Word w of a tile bitset shifted so that bit L moves to L + d (bits shifted in are 0).
TS_DEVINL uint32_t shifted_word(const uint32_t* src, int mw, int w, int d) {
    int base = 32 * w - d;
    int ws = base >> 5, bs = base & 31;
    uint32_t lo = (ws >= 0 && ws < mw) ? src[ws] : 0u;
    if (bs == 0) return lo;
    uint32_t hi = (ws + 1 >= 0 && ws + 1 < mw) ? src[ws + 1] : 0u;
    return (lo >> bs) | (hi << (32 - bs));
}

// Processes one tile of one field for sweep ordering `dir`. Returns the node evaluations made.
//
// Due nodes are tracked per node, as the reference's dirty flags do (EikonalOpenCl.cs:528-532,
// 608-622): only due nodes are evaluated (a node that is not due would get the value it holds), a
// node is no longer due once evaluated, and a node that changes makes its 12 stencil neighbours due
// — inside the tile through the wake masks after each plane, in the neighbour tiles at the end.
template <typename Real, class S, bool VARZ>
TS_DEVINL int process_tile(const Args<Real>& a, const GridDesc& g, const FieldDesc<Real>& fd, int f, int tx, int ty,
                           int tz, int dir, bool second, Real* cube, Real* ss, Real* mwx, Real* mwy, Real* mzc,
                           uint32_t* fixedm, uint32_t* dm, uint32_t* chg, uint32_t* chg_all, const uint16_t* ptab,
                           const int* poff, const uint32_t* wake, int lane) {
    const Real inf = real_inf<Real>();
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t nxy = int64_t(nx) * ny;
    const int x0 = tx * S::BX, y0 = ty * S::BY, z0 = tz * S::BZ;
    const int tid = (tz * g.ty + ty) * g.tx + tx;
    Real* __restrict__ T = fd.T;
    const Real* __restrict__ slow = fd.s;
    const bool partial = x0 + S::BX > nx || y0 + S::BY > ny || z0 + S::BZ > nz;

    // Axis weights of the tile's rows.
    const Real* wx = static_cast<const Real*>(g.wx);
    const Real* wy = static_cast<const Real*>(g.wy);
    for (int q = lane; q < 2 * S::BY * S::BZ; q += 32) {
        int r = q >> 1, j = y0 + r % S::BY, k = z0 + r / S::BY;
        mwx[q] = (j < ny && k < nz) ? ldg_r(&wx[2 * (int64_t(k) * ny + j) + (q & 1)]) : Real(1);
    }
    for (int q = lane; q < 2 * S::BZ; q += 32) mwy[q] = (z0 + (q >> 1) < nz) ? ldg_r(&wy[2 * z0 + q]) : Real(1);
    if (VARZ) {
        const Real* zc = static_cast<const Real*>(g.zc);
        for (int q = lane; q < kZCoef * S::BZ; q += 32) {
            int k = z0 + q / kZCoef;
            mzc[q] = k < nz ? ldg_r(&zc[int64_t(k) * kZCoef + q % kZCoef]) : Real(1);
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
        const bool in_range = tid >= fd.seed_tile_lo && tid <= fd.seed_tile_hi;
        int lo = 0, hi = in_range ? fd.seed_count : 0;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (__ldg(&a.seed_tile[fd.seed_begin + mid]) < tid) lo = mid + 1;
            else hi = mid;
        }
        bool has = in_range && lo < fd.seed_count && __ldg(&a.seed_tile[fd.seed_begin + lo]) == tid;
        for (int q = lane; q < S::MW; q += 32) {
            uint32_t fx = has ? __ldg(&a.seed_mask[int64_t(fd.seed_begin + lo) * S::MW + q]) : 0u;
            // Nodes off the grid (a partial tile) are treated as fixed: never evaluated, never due.
            if (partial) {
                for (int b = 0; b < 32; b++) {
                    int L = 32 * q + b;
                    int i = L % S::BX, j = (L / S::BX) % S::BY, k = L / (S::BX * S::BY);
                    if (L >= S::N || x0 + i >= nx || y0 + j >= ny || z0 + k >= nz) fx |= 1u << b;
                }
            }
            fixedm[q] = fx;
            dm[q] = __ldcg(&fd.dmask[int64_t(tid) * S::MW + q]) & ~fx;
            chg[q] = 0u;
            chg_all[q] = 0u;
        }
    }
    if (lane == 0) __stcg(&fd.dirty[tid], (uint8_t)0);
    cp_async_wait_all();
    __syncwarp();

    // Node planes of the tile in the mirrored order of `dir`; only due nodes are evaluated.
    const Real tol = a.tol;
    bool big = false, modified = false;
    int evals = 0;
    for (int p = 0; p < S::NPLANES; p++) {
        const int e0 = poff[p], e1 = poff[p + 1];
        bool changed_here = false;
        for (int eb = e0; eb < e1; eb += 32) {
            int e = eb + lane;
            int L = 0, i = 0, j = 0, k = 0;
            bool due = false;
            if (e < e1) {
                unsigned pk = ptab[e];
                int ip = pk & 31, jp = (pk >> 5) & 31, kp = pk >> 10;
                i = (dir & 1) ? S::BX - 1 - ip : ip;
                j = (dir & 2) ? S::BY - 1 - jp : jp;
                k = (dir & 4) ? S::BZ - 1 - kp : kp;
                L = (k * S::BY + j) * S::BX + i;
                due = (dm[L >> 5] >> (L & 31)) & 1u;
            }
            if (!__any_sync(0xffffffffu, due)) continue;
            if (due) {
                atomicAnd(&dm[L >> 5], ~(1u << (L & 31)));
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
                    modified = true;
                    if (counts_as_change<Real>(cur, cand, tol)) big = true;
                    if (wakes<Real>(cur, cand, a.wake_rel)) {
                        if (a.causal) {
                            // Wake each stencil neighbour holding more than cand, now: in this tile
                            // through its due mask, in a neighbour tile (whose values are the
                            // cube's halo, fixed in this visit) through the tile's global mask.
                            const int pos[3] = {i, j, k};
                            const int B[3] = {S::BX, S::BY, S::BZ};
                            const int cstep[3] = {1, S::CX, S::CX * S::CY};
                            const int nstep[3] = {1, S::BX, S::BX * S::BY};
                            const int tpos[3] = {tx, ty, tz};
                            const int tcnt[3] = {g.tx, g.ty, g.tz};
                            const int tstep[3] = {1, g.tx, g.tx * g.ty};
#pragma unroll
                            for (int ax = 0; ax < 3; ax++) {
#pragma unroll
                                for (int dd = -2; dd <= 2; dd++) {
                                    if (dd == 0) continue;
                                    if (!(cand < cube[c + dd * cstep[ax]])) continue;
                                    const int np = pos[ax] + dd;
                                    if (np >= 0 && np < B[ax]) {
                                        const int nL = L + dd * nstep[ax];
                                        if (!((fixedm[nL >> 5] >> (nL & 31)) & 1u)) atomicOr(&dm[nL >> 5], 1u << (nL & 31));
                                    } else {
                                        const int nt = np < 0 ? tpos[ax] - 1 : tpos[ax] + 1;
                                        if (nt < 0 || nt >= tcnt[ax]) continue;
                                        const int nL = L + ((np < 0 ? np + B[ax] : np - B[ax]) - pos[ax]) * nstep[ax];
                                        const int ntid = tid + (nt - tpos[ax]) * tstep[ax];
                                        atomicOr(&fd.dmask[int64_t(ntid) * S::MW + (nL >> 5)], 1u << (nL & 31));
                                        __stcg(&fd.dirty[ntid], (uint8_t)1);
                                    }
                                }
                            }
                        } else {
                            atomicOr(&chg[L >> 5], 1u << (L & 31));
                            changed_here = true;
                        }
                    }
                }
            }
        }
        // Wake the stencil neighbours of this plane's changed nodes (they lie on other planes).
        if (__any_sync(0xffffffffu, changed_here)) {
            __syncwarp();
            uint32_t wake_w = 0, c_w = 0;
            if (lane < S::MW) {
                c_w = chg[lane];
#pragma unroll
                for (int d = 0; d < 12; d++)
                    wake_w |= shifted_word(chg, S::MW, lane, stencil_offset<S>(d)) & wake[d * S::MW + lane];
            }
            __syncwarp();
            if (lane < S::MW) {
                dm[lane] |= wake_w & ~fixedm[lane];
                chg_all[lane] |= c_w;
                chg[lane] = 0u;
            }
        }
        __syncwarp();
    }
    // Hand the due nodes back; wake nodes of the neighbour tiles within two nodes of a change.
    bool any_due = false, any_chg = false;
    if (lane < S::MW) {
        uint32_t d = dm[lane] & ~fixedm[lane];
        __stcg(&fd.dmask[int64_t(tid) * S::MW + lane], d);
        any_due = d != 0u;
        any_chg = chg_all[lane] != 0u;
    }
    any_due = __any_sync(0xffffffffu, any_due);
    any_chg = __any_sync(0xffffffffu, any_chg);
    if (lane == 0 && any_due) __stcg(&fd.dirty[tid], (uint8_t)1);
    if (__any_sync(0xffffffffu, modified)) {
        for (int q = lane; q < S::N; q += 32) {
            int i = q % S::BX, j = (q / S::BX) % S::BY, k = q / (S::BX * S::BY);
            int gx = x0 + i, gy = y0 + j, gz = z0 + k;
            if (gx < nx && gy < ny && gz < nz) st_cg(&T[(int64_t(gz) * ny + gy) * pitch + S::HX + gx], cube[S::cidx(i, j, k)]);
        }
    }
    if (any_chg) {
        for (int q = lane; q < S::N; q += 32) {
            int i = q % S::BX, j = (q / S::BX) % S::BY, k = q / (S::BX * S::BY);
            if (!((chg_all[q >> 5] >> (q & 31)) & 1u)) continue;
            // Neighbours at distance 1 and 2 across each face, in the neighbour tile's coordinates.
#pragma unroll
            for (int axis = 0; axis < 3; axis++) {
                const int pos = axis == 0 ? i : axis == 1 ? j : k;
                const int B = axis == 0 ? S::BX : axis == 1 ? S::BY : S::BZ;
                const int tpos = axis == 0 ? tx : axis == 1 ? ty : tz;
                const int tcount = axis == 0 ? g.tx : axis == 1 ? g.ty : g.tz;
                const int tstride = axis == 0 ? 1 : axis == 1 ? g.tx : g.tx * g.ty;
                const int nstride = axis == 0 ? 1 : axis == 1 ? S::BX : S::BX * S::BY;
#pragma unroll
                for (int dd = -2; dd <= 2; dd++) {
                    if (dd == 0) continue;
                    int np = pos + dd;
                    if (np >= 0 && np < B) continue;  // inside this tile: woken already
                    int nt = np < 0 ? tpos - 1 : tpos + 1;
                    if (nt < 0 || nt >= tcount) continue;
                    int local = np < 0 ? np + B : np - B;
                    int nL = q + (local - pos) * nstride;
                    int ntid = tid + (nt - tpos) * tstride;
                    atomicOr(&fd.dmask[int64_t(ntid) * S::MW + (nL >> 5)], 1u << (nL & 31));
                    __stcg(&fd.dirty[ntid], (uint8_t)1);
                }
            }
        }
    }
    big = __any_sync(0xffffffffu, big);
    if (lane == 0 && big) __stcg(&a.fields[f].state->changed, 1);  // every writer writes 1
    __syncwarp();
    return evals;
}

}  // namespace eik
}  // namespace ts
