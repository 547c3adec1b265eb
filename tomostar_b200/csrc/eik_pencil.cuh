// The pencil tile of the engine: BX×8×4 nodes swept by one warp with one lane per (y, z) row.
//
// Inside a tile the reference's plane order i'+j'+k' = p (mirrored coordinates) is kept: at step p
// the lane of canonical row (j', k') evaluates the node i' = p − j' − k', so every plane of the tile
// is one step of the warp and a step holds up to 32 nodes of the plane. Each lane keeps the five
// values i'−2..i'+2 of its own row in registers (a window sliding one node per step); the values of
// the y and z neighbours at i' come from the lanes of the neighbouring rows by warp shuffles — the
// lane one row back has just evaluated that node (its window offset −1), the lane one row ahead has
// not yet (offset +1), and likewise two rows away (offsets ∓2). Rows outside the tile (the two-node
// halo on the y and z faces) are staged in shared memory once per visit. The visiting order is one
// in which every node follows its axis neighbours of smaller p, so the field is the reference's to
// the bit, as for the other tile shapes.
//
// Due nodes are tracked per node as the reference's dirty flags (EikonalOpenCl.cs:528-532,
// 608-622): one 64-bit row mask per lane; a changed node wakes its x neighbours in the lane's own
// mask, and its y and z neighbours through one ballot of the changed lanes per step.
#pragma once

#include <type_traits>

#include "eik_kernels.cuh"

namespace ts {
namespace eik {

constexpr int kPencilBY = 8, kPencilBZ = 4;

// Shared memory of one warp: the 48 halo rows of the tile, BX values each in grid x order —
// 16 y rows (canonical j' = −2, −1, 8, 9 for each k') then 32 z rows (k' = −2, −1, 4, 5 for each j').
template <typename Real, int BX>
struct PencilSmem {
    static constexpr int kRows = 16 + 32;
    static constexpr int kBytes = kRows * BX * int(sizeof(Real));
};

// Halo row of canonical row c (< 0 or >= B on its axis): slot 0..3 for c = −2, −1, B, B+1.
TS_HDINL int halo_slot(int c, int B) { return c < 0 ? c + 2 : c - B + 2; }

// One bit per node of a row: 64-bit words for 64-wide pencils, 32-bit for 32-wide ones.
template <int BX>
using RowMask = std::conditional_t<BX == 64, uint64_t, uint32_t>;

template <int BX>
TS_DEVINL RowMask<BX> row_reverse(RowMask<BX> m) {
    if constexpr (BX == 64) return __brevll(m);
    else return __brev(m);
}

// Variants of the visit (OPT bits): kRing2 — a two-deep prefetch ring instead of four;
// kLazyW — axis weights read where an update uses them instead of held in registers for the visit.
// Both only trade registers (the values computed are the same).
// kSpecAll — the sweep ordering fixed at compile time whatever the width and occupancy (lockstep).
// kReshuffle — the y and z neighbour values are fetched again for the wake tests after an update
// instead of being held through it (within a step no lane changes the window values it shares).
constexpr int kRing2 = 1, kLazyW = 2, kSpecAll = 4, kReshuffle = 8;

template <typename Real, int BX, bool VARZ, int SDIR, int OPT = 0>
TS_DEVINL int process_pencil(const Args<Real>& a, const GridDesc& g, const FieldDesc<Real>& fd, int f, int tx, int ty,
                             int tz, int dir, bool second, Real* halo, int lane);

// The pencil visit with the sweep ordering specialised where that pays (SPEC): FP64 pencils whose
// launch leaves room for the extra registers (64-wide pencils, and 32-wide ones at 12 warps per SM),
// under the lockstep scheduler, where every warp of a step runs the same ordering.
template <typename Real, int BX, bool VARZ, bool SPEC, int OPT = 0>
TS_DEVINL int visit_pencil(const Args<Real>& a, const GridDesc& g, const FieldDesc<Real>& fd, int f, int tx, int ty,
                           int tz, int dir, bool second, Real* halo, int lane) {
    if constexpr (SPEC && is_f64<Real>()) {
        switch (dir) {
#define TS_PENCIL_DIR(d) \
    case d: return process_pencil<Real, BX, VARZ, d, OPT>(a, g, fd, f, tx, ty, tz, dir, second, halo, lane);
            TS_PENCIL_DIR(0) TS_PENCIL_DIR(1) TS_PENCIL_DIR(2) TS_PENCIL_DIR(3)
            TS_PENCIL_DIR(4) TS_PENCIL_DIR(5) TS_PENCIL_DIR(6) TS_PENCIL_DIR(7)
#undef TS_PENCIL_DIR
        }
        return 0;
    } else {
        return process_pencil<Real, BX, VARZ, -1, OPT>(a, g, fd, f, tx, ty, tz, dir, second, halo, lane);
    }
}

// SDIR 0..7: the sweep ordering fixed at compile time, so that the mirroring costs nothing in the
// step loop (used for 64-wide FP64 pencils); −1: read from dir at run time (32-wide pencils, where
// the specialised code needs more registers than the 128 their occupancy allows, and FP32).
template <typename Real, int BX, bool VARZ, int SDIR, int OPT>
TS_DEVINL int process_pencil(const Args<Real>& a, const GridDesc& g, const FieldDesc<Real>& fd, int f, int tx, int ty,
                             int tz, int dir, bool second, Real* halo, int lane) {
    static_assert(BX == 32 || BX == 64, "pencil rows are 32 or 64 nodes");
    constexpr int RING = (OPT & kRing2) ? 2 : 4;  // prefetch depth (steps ahead)
    constexpr bool LAZYW = (OPT & kLazyW) != 0;
    constexpr bool RESHUFFLE = (OPT & kReshuffle) != 0;
    constexpr int BY = kPencilBY, BZ = kPencilBZ, HX = Layout<Real>::HX;
    constexpr int MWR = BX / 32;           // mask words per row
    constexpr int MW = BX * BY * BZ / 32;  // mask words per tile
    constexpr unsigned FULL = 0xffffffffu;
    using Mask = RowMask<BX>;
    constexpr Mask kOne = 1;
    constexpr Mask kRowBits = Mask(~Mask(0));
    const Real inf = real_inf<Real>();
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int x0 = tx * BX, y0 = ty * BY, z0 = tz * BZ;
    const int tid = (tz * g.ty + ty) * g.tx + tx;
    const int sd = SDIR < 0 ? dir : SDIR;
    const bool mx = (sd & 1) != 0, my = (sd & 2) != 0, mz = (sd & 4) != 0;
    const int jp = lane & 7, kp = lane >> 3;  // canonical row of the lane
    const int j = my ? BY - 1 - jp : jp, k = mz ? BZ - 1 - kp : kp;
    const int gy = y0 + j, gz = z0 + k;
    const bool row_on = gy < ny && gz < nz;
    const int pitch = g.pitch;
    const int64_t rowi = int64_t(gz) * ny + gy;
    Real* __restrict__ row = fd.T + rowi * pitch + HX + x0;  // dereferenced only when row_on
    const Real* __restrict__ srow = fd.s + rowi * nx + x0;

    // Halo rows → shared memory (16-byte copies in grid x order; +inf for rows off the grid).
    {
        constexpr int NCH = BX * int(sizeof(Real)) / 16;
        constexpr int PER = 16 / int(sizeof(Real));
        for (int q = lane; q < 48 * NCH; q += 32) {
            const int h = q / NCH, ch = q - h * NCH;
            int hj, hk;  // canonical row of halo row h
            if (h < 16) {
                const int slot = h >> 2;
                hj = slot < 2 ? slot - 2 : slot - 2 + BY;
                hk = h & 3;
            } else {
                const int slot = (h - 16) >> 3;
                hk = slot < 2 ? slot - 2 : slot - 2 + BZ;
                hj = (h - 16) & 7;
            }
            const int ay = y0 + (my ? BY - 1 - hj : hj), az = z0 + (mz ? BZ - 1 - hk : hk);
            Real* dst = halo + h * BX + ch * PER;
            if (ay >= 0 && ay < ny && az >= 0 && az < nz) {
                cp_async16_cg(dst, fd.T + (int64_t(az) * ny + ay) * pitch + HX + x0 + ch * PER);
            } else {
#pragma unroll
                for (int e = 0; e < PER; e++) dst[e] = inf;
            }
        }
    }
    // Shared-memory rows of the eight neighbour directions that leave the tile (−1: a lane's shuffle).
    auto yhalo = [&](int c) { return (c < 0 || c >= BY) ? (halo_slot(c, BY) * 4 + kp) * BX : -1; };
    auto zhalo = [&](int c) { return (c < 0 || c >= BZ) ? (16 + halo_slot(c, BZ) * 8 + jp) * BX : -1; };
    const int hy_m1 = yhalo(jp - 1), hy_p1 = yhalo(jp + 1), hy_m2 = yhalo(jp - 2), hy_p2 = yhalo(jp + 2);
    const int hz_m1 = zhalo(kp - 1), hz_p1 = zhalo(kp + 1), hz_m2 = zhalo(kp - 2), hz_p2 = zhalo(kp + 2);

    // The lane's row: weights, fixed (seed or off-grid) and due nodes, in canonical x order.
    const Real* wxp = static_cast<const Real*>(g.wx);
    const Real* wyp = static_cast<const Real*>(g.wy);
    Real wx1 = Real(1), wx2 = Real(1), wy1 = Real(1), wy2 = Real(1);
    if (row_on && !LAZYW) {
        wx1 = ldg_r(&wxp[2 * rowi]);
        wx2 = ldg_r(&wxp[2 * rowi + 1]);
        wy1 = ldg_r(&wyp[2 * gz]);
        wy2 = ldg_r(&wyp[2 * gz + 1]);
    }
    const Real wz1 = Real(g.wz1), wz2 = Real(g.wz2);
    const Real* zc = VARZ ? static_cast<const Real*>(g.zc) + kZCoef * (row_on ? gz : 0) : nullptr;
    const int r = k * BY + j;
    Mask fixed = 0, due = 0;
    {
        const bool in_range = tid >= fd.seed_tile_lo && tid <= fd.seed_tile_hi;
        int lo = 0, hi = in_range ? fd.seed_count : 0;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (__ldg(&a.seed_tile[fd.seed_begin + mid]) < tid) lo = mid + 1;
            else hi = mid;
        }
        const bool has = in_range && lo < fd.seed_count && __ldg(&a.seed_tile[fd.seed_begin + lo]) == tid;
        Mask fx = 0, dm = 0;
#pragma unroll
        for (int w = 0; w < MWR; w++) {
            if (has) fx |= Mask(__ldg(&a.seed_mask[int64_t(fd.seed_begin + lo) * MW + r * MWR + w])) << (32 * w);
            dm |= Mask(__ldcg(&fd.dmask[int64_t(tid) * MW + r * MWR + w])) << (32 * w);
        }
        if (!row_on) fx = kRowBits;
        else if (x0 + BX > nx) fx |= kRowBits & ~((kOne << (nx - x0)) - kOne);  // x off the grid
        fixed = mx ? row_reverse<BX>(fx) : fx;
        due = (mx ? row_reverse<BX>(dm) : dm) & ~fixed;
    }
    if (lane == 0) __stcg(&fd.dirty[tid], (uint8_t)0);

    // Window and prefetch rings. Canonical x c ↦ grid x offset ax(c); the row's pads (and the
    // tile's nodes beyond nx) hold +inf, so x needs no check inside [−2, BX+1].
    // Positions outside [−2, BX+1] (times) or off the grid (slowness) are clamped to a valid address:
    // those values only ever fill window slots that no evaluation and no neighbour lane reads.
    auto ax = [&](int c) { return mx ? BX - 1 - c : c; };
    [[maybe_unused]] const int xlast = min(BX, nx - x0) - 1;  // last on-grid x offset of the tile
    auto ldT = [&](int c) -> Real {
        if constexpr (SDIR >= 0) return row_on ? ld_cg(row + ax(max(-2, min(c, BX + 1)))) : inf;
        else return (row_on && c >= -2 && c <= BX + 1) ? ld_cg(row + ax(c)) : inf;
    };
    auto ldS = [&](int c) -> Real {
        if constexpr (SDIR >= 0) return row_on ? ldg_r(srow + max(0, min(ax(c), xlast))) : Real(0);
        else return (row_on && c >= 0 && c < BX && x0 + ax(c) < nx) ? ldg_r(srow + ax(c)) : Real(0);
    };
    const int ip0 = -jp - kp;
    Real W0 = ldT(ip0 - 2), W1 = ldT(ip0 - 1), W2 = ldT(ip0), W3 = ldT(ip0 + 1), W4 = ldT(ip0 + 2);
    Real tr[RING], sr[RING];
#pragma unroll
    for (int u = 0; u < RING; u++) {
        tr[u] = ldT(ip0 + 3 + u);
        sr[u] = ldS(ip0 + u);
    }
    cp_async_wait_all();
    __syncwarp();

    const Real tol = a.tol, wake_rel = a.wake_rel;
    const bool causal = a.causal != 0;
    auto bit = [](int c) -> Mask { return (unsigned)c < unsigned(BX) ? Mask(kOne << c) : Mask(0); };
    // Woken nodes of the neighbour tiles, as row masks in canonical x: the rows one and two beyond
    // the lane's own y and z faces (a lane has at most one such side per axis), and the x halo.
    Mask wky1 = 0, wky2 = 0, wkz1 = 0, wkz2 = 0;
    unsigned wxh = 0;  // bits 0..3: canonical x = −1, −2, BX, BX+1
    bool big = false;
    int evals = 0;
    constexpr int NSTEPS = (BX + BY + BZ - 2 + RING - 1) / RING * RING;
    for (int p0 = 0; p0 < NSTEPS; p0 += RING) {
#pragma unroll
        for (int u = 0; u < RING; u++) {
            const int ip = p0 + u + ip0;
            const bool is_due = (due >> (ip & (BX - 1))) & (unsigned(ip) < unsigned(BX));
            if (__any_sync(FULL, is_due)) {
                // Canonical neighbours: one row back has evaluated this x (its offset −1), one row
                // ahead has not (offset +1); two rows away likewise at offsets ∓2.
                Real yb1 = shfl_up_r(FULL, W1, 1), ya1 = shfl_down_r(FULL, W3, 1);
                Real yb2 = shfl_up_r(FULL, W0, 2), ya2 = shfl_down_r(FULL, W4, 2);
                Real zb1 = shfl_up_r(FULL, W1, 8), za1 = shfl_down_r(FULL, W3, 8);
                Real zb2 = shfl_up_r(FULL, W0, 16), za2 = shfl_down_r(FULL, W4, 16);
                bool chg = false;
                if (is_due) {
                    const int x = ax(ip);
                    if (hy_m1 >= 0) yb1 = halo[hy_m1 + x];
                    if (hy_p1 >= 0) ya1 = halo[hy_p1 + x];
                    if (hy_m2 >= 0) yb2 = halo[hy_m2 + x];
                    if (hy_p2 >= 0) ya2 = halo[hy_p2 + x];
                    if (hz_m1 >= 0) zb1 = halo[hz_m1 + x];
                    if (hz_p1 >= 0) za1 = halo[hz_p1 + x];
                    if (hz_m2 >= 0) zb2 = halo[hz_m2 + x];
                    if (hz_p2 >= 0) za2 = halo[hz_p2 + x];
                    due &= ~(kOne << ip);
                    evals++;
                    // Canonical → grid orientation (minus = smaller grid index).
                    const Real xm = mx ? W3 : W1, xp = mx ? W1 : W3, xm2 = mx ? W4 : W0, xp2 = mx ? W0 : W4;
                    const Real ym = my ? ya1 : yb1, yp = my ? yb1 : ya1, ym2 = my ? ya2 : yb2, yp2 = my ? yb2 : ya2;
                    const Real zm = mz ? za1 : zb1, zp = mz ? zb1 : za1, zm2 = mz ? za2 : zb2, zp2 = mz ? zb2 : za2;
                    if constexpr (LAZYW) {  // due lanes lie on the grid (off-grid rows are fixed)
                        wx1 = ldg_r(&wxp[2 * rowi]);
                        wx2 = ldg_r(&wxp[2 * rowi + 1]);
                        wy1 = ldg_r(&wyp[2 * gz]);
                        wy2 = ldg_r(&wyp[2 * gz + 1]);
                    }
                    const Real cand = Update<Real, VARZ>::eval(sr[u], xm, xp, xm2, xp2, ym, yp, ym2, yp2, zm, zp, zm2,
                                                               zp2, wx1, wx2, wy1, wy2, wz1, wz2, zc, second);
                    if (cand < W2) {
                        if (counts_as_change<Real>(W2, cand, tol)) big = true;
                        chg = wakes<Real>(W2, cand, wake_rel);
                        W2 = cand;
                        st_cg(row + x, cand);
                    }
                }
                const unsigned cb = __ballot_sync(FULL, chg);
                if (cb) {
                    if constexpr (RESHUFFLE) {
                        yb1 = shfl_up_r(FULL, W1, 1);
                        ya1 = shfl_down_r(FULL, W3, 1);
                        yb2 = shfl_up_r(FULL, W0, 2);
                        ya2 = shfl_down_r(FULL, W4, 2);
                        zb1 = shfl_up_r(FULL, W1, 8);
                        za1 = shfl_down_r(FULL, W3, 8);
                        zb2 = shfl_up_r(FULL, W0, 16);
                        za2 = shfl_down_r(FULL, W4, 16);
                        if (chg) {
                            const int x = ax(ip);
                            if (hy_m1 >= 0) yb1 = halo[hy_m1 + x];
                            if (hy_p1 >= 0) ya1 = halo[hy_p1 + x];
                            if (hy_m2 >= 0) yb2 = halo[hy_m2 + x];
                            if (hy_p2 >= 0) ya2 = halo[hy_p2 + x];
                            if (hz_m1 >= 0) zb1 = halo[hz_m1 + x];
                            if (hz_p1 >= 0) za1 = halo[hz_p1 + x];
                            if (hz_m2 >= 0) zb2 = halo[hz_m2 + x];
                            if (hz_p2 >= 0) za2 = halo[hz_p2 + x];
                        }
                    }
                    // A changed node wakes its 12 stencil neighbours (with the causal rule, those
                    // holding more than its new value W2). The y and z neighbours are woken through
                    // one ballot per direction: a change one row back wakes x = i'+1 of this row,
                    // one row ahead x = i'−1, and two rows back or ahead x = i'±2.
                    auto wk_if = [&](Real v) { return chg && (!causal || W2 < v); };
                    Mask wk = 0;
                    if (wk_if(W1)) wk |= bit(ip - 1);
                    if (wk_if(W3)) wk |= bit(ip + 1);
                    if (wk_if(W0)) wk |= bit(ip - 2);
                    if (wk_if(W4)) wk |= bit(ip + 2);
                    // Without the causal rule every direction's ballot is the ballot of the changes.
                    unsigned Byb1 = cb, Bya1 = cb, Byb2 = cb, Bya2 = cb, Bzb1 = cb, Bza1 = cb, Bzb2 = cb, Bza2 = cb;
                    if (causal) {  // the same for the whole warp
                        Byb1 = __ballot_sync(FULL, wk_if(yb1));
                        Bya1 = __ballot_sync(FULL, wk_if(ya1));
                        Byb2 = __ballot_sync(FULL, wk_if(yb2));
                        Bya2 = __ballot_sync(FULL, wk_if(ya2));
                        Bzb1 = __ballot_sync(FULL, wk_if(zb1));
                        Bza1 = __ballot_sync(FULL, wk_if(za1));
                        Bzb2 = __ballot_sync(FULL, wk_if(zb2));
                        Bza2 = __ballot_sync(FULL, wk_if(za2));
                    }
                    if ((jp >= 1 && ((Bya1 >> (lane - 1)) & 1u)) || (kp >= 1 && ((Bza1 >> (lane - 8)) & 1u)))
                        wk |= bit(ip + 1);
                    if ((jp <= BY - 2 && ((Byb1 >> (lane + 1)) & 1u)) || (kp <= BZ - 2 && ((Bzb1 >> (lane + 8)) & 1u)))
                        wk |= bit(ip - 1);
                    if ((jp >= 2 && ((Bya2 >> (lane - 2)) & 1u)) || (kp >= 2 && ((Bza2 >> (lane - 16)) & 1u)))
                        wk |= bit(ip + 2);
                    if ((jp <= BY - 3 && ((Byb2 >> (lane + 2)) & 1u)) || (kp <= BZ - 3 && ((Bzb2 >> (lane + 16)) & 1u)))
                        wk |= bit(ip - 2);
                    due |= wk & ~fixed;
                    if (chg) {
                        // Neighbours in other tiles (their values are the halo's, fixed in this visit).
                        const Mask b = kOne << ip;
                        if ((hy_m1 >= 0 && wk_if(yb1)) || (hy_p1 >= 0 && wk_if(ya1))) wky1 |= b;
                        if ((hy_m2 >= 0 && wk_if(yb2)) || (hy_p2 >= 0 && wk_if(ya2))) wky2 |= b;
                        if ((hz_m1 >= 0 && wk_if(zb1)) || (hz_p1 >= 0 && wk_if(za1))) wkz1 |= b;
                        if ((hz_m2 >= 0 && wk_if(zb2)) || (hz_p2 >= 0 && wk_if(za2))) wkz2 |= b;
                        if (ip == 0 && wk_if(W1)) wxh |= 1u;
                        if (ip <= 1 && wk_if(W0)) wxh |= ip == 0 ? 2u : 1u;
                        if (ip == BX - 1 && wk_if(W3)) wxh |= 4u;
                        if (ip >= BX - 2 && wk_if(W4)) wxh |= ip == BX - 1 ? 8u : 4u;
                    }
                }
            }
            // Slide the window one node and refill the rings four nodes ahead.
            W0 = W1;
            W1 = W2;
            W2 = W3;
            W3 = W4;
            W4 = tr[u];
            tr[u] = ldT(ip + 3 + RING);
            sr[u] = ldS(ip + RING);
        }
    }

    // Hand the due nodes back; wake the nodes of the neighbour tiles within two nodes of a change.
    const Mask due_g = mx ? row_reverse<BX>(due & ~fixed) : Mask(due & ~fixed);
#pragma unroll
    for (int w = 0; w < MWR; w++) __stcg(&fd.dmask[int64_t(tid) * MW + r * MWR + w], uint32_t(due_g >> (32 * w)));
    if (__any_sync(FULL, due_g != 0) && lane == 0) __stcg(&fd.dirty[tid], (uint8_t)1);
    auto wake_row = [&](int ntid, int nr, Mask canon_bits) {
        const Mask bits = mx ? row_reverse<BX>(canon_bits) : canon_bits;
#pragma unroll
        for (int w = 0; w < MWR; w++) {
            const uint32_t m = uint32_t(bits >> (32 * w));
            if (m) atomicOr(&fd.dmask[int64_t(ntid) * MW + nr * MWR + w], m);
        }
        __stcg(&fd.dirty[ntid], (uint8_t)1);
    };
    // Rows beyond the y and z faces: canonical row c outside the tile → the neighbour tile and its row.
    auto wake_y = [&](int c, Mask bits) {
        if (!bits) return;
        int ay = my ? BY - 1 - c : c;  // tile-local actual row, outside [0, BY)
        int nty = ay < 0 ? ty - 1 : ty + 1;
        if (nty < 0 || nty >= g.ty) return;
        wake_row(tid + (nty - ty) * g.tx, k * BY + (ay < 0 ? ay + BY : ay - BY), bits);
    };
    auto wake_z = [&](int c, Mask bits) {
        if (!bits) return;
        int az = mz ? BZ - 1 - c : c;
        int ntz = az < 0 ? tz - 1 : tz + 1;
        if (ntz < 0 || ntz >= g.tz) return;
        wake_row(tid + (ntz - tz) * g.tx * g.ty, (az < 0 ? az + BZ : az - BZ) * BY + j, bits);
    };
    wake_y(jp == 0 ? -1 : BY, wky1);                      // one row beyond (lanes j' = 0, BY − 1)
    wake_y(jp <= 1 ? jp - 2 : jp + 2, wky2);              // two rows beyond (j' = 0, 1, BY − 2, BY − 1)
    wake_z(kp == 0 ? -1 : BZ, wkz1);
    wake_z(kp <= 1 ? kp - 2 : kp + 2, wkz2);
    if (wxh) {
        // Canonical x −1, −2 lie in the tile before along the sweep, BX, BX+1 in the one after.
        const int back = mx ? tx + 1 : tx - 1, ahead = mx ? tx - 1 : tx + 1;
        const Mask top = kOne << (BX - 1), top2 = kOne << (BX - 2);
        // In the neighbour tile's canonical x, −1 ↦ BX−1, −2 ↦ BX−2, BX ↦ 0, BX+1 ↦ 1.
        if ((wxh & 3u) && back >= 0 && back < g.tx)
            wake_row(tid + (back - tx), r, Mask(((wxh & 1u) ? top : Mask(0)) | ((wxh & 2u) ? top2 : Mask(0))));
        if ((wxh & 12u) && ahead >= 0 && ahead < g.tx)
            wake_row(tid + (ahead - tx), r, Mask(((wxh & 4u) ? 1u : 0u) | ((wxh & 8u) ? 2u : 0u)));
    }
    big = __any_sync(FULL, big);
    if (lane == 0 && big) __stcg(&a.fields[f].state->changed, 1);  // every writer writes 1
    __syncwarp();
    return evals;
}

}  // namespace eik
}  // namespace ts
