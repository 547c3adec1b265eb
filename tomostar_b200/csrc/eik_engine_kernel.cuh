// The engine's cooperative persistent kernel: diagonal steps over every running field's tiles,
// round ends, and phase changes, in one launch.
#pragma once

#include "eik_kernels.cuh"
#include "eik_pencil.cuh"

namespace ts {
namespace eik {

// PENCIL: BX×8×4 tiles swept by process_pencil (one lane per row); otherwise cube tiles swept by
// process_tile (node planes with a plane table).
template <typename Real, int BX, int BY, int BZ, int WARPS, int MINB, bool VARZ_ANY, bool PENCIL, int OPT = 0>
__global__ void __launch_bounds__(WARPS * 32, MINB) engine_kernel(Args<Real> a) {
    using S = Shape<Real, BX, BY, BZ>;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int kWarpBytes = PENCIL ? PencilSmem<Real, BX>::kBytes : WarpSmem<Real, S>::kBytes;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* mine = smem + warp * kWarpBytes;
    Real* cube = reinterpret_cast<Real*>(mine);
    Real* ss = cube + S::CUBE;
    Real* mwx = ss + S::N;
    Real* mwy = mwx + 2 * S::BY * S::BZ;
    Real* mzc = mwy + 2 * S::BZ;
    uint32_t* fixedm = reinterpret_cast<uint32_t*>(mzc + kZCoef * S::BZ);
    uint32_t* dm = fixedm + S::MW;
    uint32_t* chg = dm + S::MW;
    uint32_t* chg_all = chg + S::MW;
    uint16_t* ptab = reinterpret_cast<uint16_t*>(smem + WARPS * kWarpBytes);
    int* poff = reinterpret_cast<int*>(smem + WARPS * kWarpBytes + (S::N * 2 + 15) / 16 * 16);
    uint32_t* wake = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(poff) +
                                                 ((S::NPLANES + 1) * 4 + 15) / 16 * 16);
    if (!PENCIL) {
        for (int q = threadIdx.x; q < S::N; q += blockDim.x) ptab[q] = a.plane_tab[q];
        for (int q = threadIdx.x; q <= S::NPLANES; q += blockDim.x) poff[q] = a.plane_off[q];
        for (int q = threadIdx.x; q < 12 * S::MW; q += blockDim.x) wake[q] = a.wake_mask[q];
    }
    __syncthreads();

    const unsigned nblocks = gridDim.x;
    const int gwarp = blockIdx.x * WARPS + warp;
    const int nwarps = nblocks * WARPS;
    const int G = a.plan.ngroups;
    unsigned long long my_updates = 0, my_visits = 0;
    int rounds_this_launch = 0;
    int step = 0;

    for (;;) {
        for (int dir = 0; dir < 8; dir++) {
            for (int q = 0; q < a.plan.maxdiag; q++) {
                const int* pre = a.plan.pre + int64_t(q) * (G + 1);
                const int total = __ldg(&pre[G]);
                // Two passes per step. First the step's items are dealt round-robin to the warps
                // (item = gwarp + j·nwarps), each lane decoding one item, and the due tiles are
                // appended to a worklist. Then the warps take worklist entries one at a time, so a
                // step ends when the work does, not when the unluckiest warp's share does.
                const int par = step & 1;
                if (blockIdx.x == 0 && threadIdx.x == 0) {  // the previous step's counters: free since its barrier
                    a.ctl->produced[par ^ 1] = 0;
                    a.ctl->consumed[par ^ 1] = 0;
                }
                unsigned long long* wl = a.worklist + int64_t(par) * a.worklist_cap;
                for (int64_t j0 = 0; gwarp + j0 * nwarps < total; j0 += 32) {
                    int64_t item64 = gwarp + (j0 + lane) * nwarps;
                    int item = item64 < total ? int(item64) : total;
                    bool due = false;
                    unsigned long long entry = 0;
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
                        int tx = (dir & 1) ? g.tx - 1 - ca : ca;
                        int ty = (dir & 2) ? g.ty - 1 - cb : cb;
                        int tz = (dir & 4) ? g.tz - 1 - cc : cc;
                        const FieldState* st = a.fields[fld].state;
                        if (*(volatile const int*)&st->status == kRunning) {
                            const FieldDesc<Real>& fd = a.fields[fld];
                            due = __ldcg(&fd.dirty[(tz * g.ty + ty) * g.tx + tx]) != 0;
                        }
                        entry = (static_cast<unsigned long long>(unsigned(fld)) << 32) | unsigned(tx) |
                                (unsigned(ty) << 10) | (unsigned(tz) << 20);
                    }
                    unsigned m = __ballot_sync(0xffffffffu, due);
                    if (m) {
                        int base = 0;
                        if (lane == 0) base = atomicAdd(&a.ctl->produced[par], __popc(m));
                        base = __shfl_sync(0xffffffffu, base, 0);
                        if (due) __stcg(&wl[base + __popc(m & ((1u << lane) - 1u))], entry);
                    }
                }
                if (!grid_barrier(a.ctl, nblocks, a.barrier_timeout_ns)) goto done;
                {
                    const int listed = *(volatile int*)&a.ctl->produced[par];
                    for (;;) {
                        int idx = 0;
                        if (lane == 0) idx = atomicAdd(&a.ctl->consumed[par], 1);
                        idx = __shfl_sync(0xffffffffu, idx, 0);
                        if (idx >= listed) break;
                        unsigned long long e = __ldcg(&wl[idx]);
                        int ff = int(e >> 32);
                        int sx = int(e & 1023u), sy = int((e >> 10) & 1023u), sz = int((e >> 20) & 1023u);
                        const FieldDesc<Real>& fd = a.fields[ff];
                        const GridDesc& g = a.grids[fd.grid];
                        bool second = *(volatile const int*)&a.fields[ff].state->phase == 1;
                        int ev;
                        if constexpr (PENCIL) {
                            Real* halo = reinterpret_cast<Real*>(mine);
                            if (VARZ_ANY && g.varz)
                                ev = visit_pencil<Real, BX, true, (BX == 64 || MINB <= 3 || (OPT & kSpecAll) != 0), OPT>(a, g, fd, ff, sx, sy, sz, dir, second, halo, lane);
                            else
                                ev = visit_pencil<Real, BX, false, (BX == 64 || MINB <= 3 || (OPT & kSpecAll) != 0), OPT>(a, g, fd, ff, sx, sy, sz, dir, second, halo, lane);
                        } else {
                            if (VARZ_ANY && g.varz)
                                ev = process_tile<Real, S, true>(a, g, fd, ff, sx, sy, sz, dir, second, cube, ss, mwx,
                                                                 mwy, mzc, fixedm, dm, chg, chg_all, ptab, poff, wake,
                                                                 lane);
                            else
                                ev = process_tile<Real, S, false>(a, g, fd, ff, sx, sy, sz, dir, second, cube, ss, mwx,
                                                                  mwy, mzc, fixedm, dm, chg, chg_all, ptab, poff, wake,
                                                                  lane);
                        }
                        my_updates += ev;
                        my_visits += 1;
                    }
                }
                step++;
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
                volatile FieldState* st = a.fields[fld].state;
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
            if (!*(volatile int*)&a.fields[fld].state->enter1) continue;
            const FieldDesc<Real>& fd = a.fields[fld];
            const GridDesc& g = a.grids[fd.grid];
            int nt = g.tx * g.ty * g.tz;
            for (int q = threadIdx.x; q < nt; q += blockDim.x) __stcg(&fd.dirty[q], (uint8_t)1);
            const int64_t words = int64_t(nt) * ((BX * BY * BZ + 31) / 32);
            for (int64_t q = threadIdx.x; q < words; q += blockDim.x) __stcg(&fd.dmask[q], 0xffffffffu);
            __syncthreads();
            if (threadIdx.x == 0) a.fields[fld].state->enter1 = 0;
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


// ---- flow scheduler: no grid-wide barrier; each field advances on its own ----------------------
//
// A field's sweep needs only that a tile diagonal q is done before diagonal q+1 of the same field
// starts (the order argument of the engine); fields are independent. So each field keeps its own
// position (ordering, diagonal) and count of outstanding tiles; its due tiles go into one global
// queue that every warp of the launch takes from. The warp that finishes a field's last tile of a
// diagonal advances that field: it finds the next diagonal with due tiles (across sweeps and round
// ends, which it evaluates for that field alone) and queues them. A launch ends when every field
// has settled, been refused at the cap, been cancelled, or run its rounds for this launch. Waits
// for a queue slot are bounded (globaltimer); a wait that runs out raises the abort flag and the
// launch ends with TS_E_TIMEOUT.

// Ends a round of field f (SphericalEikonal.cs:297-323; EikonalOpenCl.cs:241-269). Whole warp.
// Returns true when the field stops in this launch.
template <typename Real, int MW>
TS_DEVINL bool flow_round_end(const Args<Real>& a, int f, int lane) {
    const FieldDesc<Real>& fd = a.fields[f];
    volatile FieldState* st = fd.state;
    bool stop = false, fill = false;
    if (lane == 0) {
        const int cap = fd.cap;
        if (!st->changed) {
            if (st->phase == 0) {
                st->rounds0 = st->round + 1;
                st->phase = 1;
                st->round = 0;
                fill = true;  // phase 1 starts with every node due (EikonalOpenCl.cs:235-239)
            } else {
                st->rounds1 = st->round + 1;
                st->status = kSettled;
                stop = true;
            }
        } else {
            st->round = st->round + 1;
            if (st->round >= cap) {
                if (st->phase == 0) st->rounds0 = st->round;
                else st->rounds1 = st->round;
                st->status = kUnsettled;
                stop = true;
            }
        }
        st->changed = 0;
        st->launch_rounds = st->launch_rounds + 1;
        if (!stop && a.max_rounds_per_launch > 0 && st->launch_rounds >= a.max_rounds_per_launch) stop = true;
        if (!stop && a.epoch_budget_ns > 0 &&
            (long long)(global_ns() - *(volatile unsigned long long*)&a.ctl->t_start) > a.epoch_budget_ns)
            stop = true;
        if (!stop && a.cancel && *a.cancel) {
            atomicCAS(&a.ctl->error, 0, TS_E_CANCELLED);
            stop = true;
        }
    }
    stop = __shfl_sync(0xffffffffu, stop, 0);
    fill = __shfl_sync(0xffffffffu, fill, 0);
    if (fill) {
        const GridDesc& g = a.grids[fd.grid];
        const int64_t nt = int64_t(g.tx) * g.ty * g.tz;
        for (int64_t q = lane; q < nt; q += 32) __stcg(&fd.dirty[q], (uint8_t)1);
        for (int64_t q = lane; q < nt * MW; q += 32) __stcg(&fd.dmask[q], 0xffffffffu);
    }
    return stop;
}

// Moves field f to its next diagonal with due tiles (from its current one, or from the start of a
// round when `start`) and queues those tiles; or stops the field. Whole warp.
template <typename Real, int MW>
TS_DEVINL void flow_advance(const Args<Real>& a, int f, bool start, int lane) {
    const FieldDesc<Real>& fd = a.fields[f];
    const GridDesc& g = a.grids[fd.grid];
    volatile FieldState* st = fd.state;
    int dir = start ? 0 : st->dir, q = start ? 0 : st->q + 1;
    for (;;) {
        if (q >= g.ndiag) {
            q = 0;
            if (++dir == 8) {
                dir = 0;
                __threadfence();
                const bool stopped = flow_round_end<Real, MW>(a, f, lane);
                __threadfence();
                __syncwarp();
                if (stopped) {
                    if (lane == 0) {
                        st->dir = 0;
                        st->q = 0;
                        st->pending = 0;
                        if (atomicSub(&a.ctl->running, 1) == 1) atomicExch(&a.ctl->done, 1);
                    }
                    __syncwarp();
                    return;
                }
            }
        }
        // Due tiles of diagonal q under ordering dir.
        const int d0 = __ldg(&g.diag_off[q]), cnt = __ldg(&g.diag_off[q + 1]) - d0;
        int due_total = 0;
        for (int b = 0; b < cnt; b += 32) {
            bool due = false;
            if (b + lane < cnt) {
                uint32_t pk = __ldg(&g.diag_tiles[d0 + b + lane]);
                int ca = pk & 1023, cb = (pk >> 10) & 1023, cc = pk >> 20;
                int tx = (dir & 1) ? g.tx - 1 - ca : ca, ty = (dir & 2) ? g.ty - 1 - cb : cb,
                    tz = (dir & 4) ? g.tz - 1 - cc : cc;
                due = __ldcg(&fd.dirty[(tz * g.ty + ty) * g.tx + tx]) != 0;
            }
            due_total += __popc(__ballot_sync(0xffffffffu, due));
        }
        if (due_total == 0) {
            q++;
            continue;
        }
        // Publish the position and count before the tiles: a consumer may finish one at once.
        if (lane == 0) {
            st->dir = dir;
            st->q = q;
            st->pending = due_total;
        }
        __syncwarp();
        __threadfence();
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&a.ctl->q_tail, (unsigned long long)due_total);
        base = __shfl_sync(0xffffffffu, base, 0);
        int written = 0;
        for (int b = 0; b < cnt; b += 32) {
            bool due = false;
            unsigned long long item = 0;
            if (b + lane < cnt) {
                uint32_t pk = __ldg(&g.diag_tiles[d0 + b + lane]);
                int ca = pk & 1023, cb = (pk >> 10) & 1023, cc = pk >> 20;
                int tx = (dir & 1) ? g.tx - 1 - ca : ca, ty = (dir & 2) ? g.ty - 1 - cb : cb,
                    tz = (dir & 4) ? g.tz - 1 - cc : cc;
                due = __ldcg(&fd.dirty[(tz * g.ty + ty) * g.tx + tx]) != 0;
                item = (static_cast<unsigned long long>(unsigned(f)) << 32) | unsigned(tx) | (unsigned(ty) << 10) |
                       (unsigned(tz) << 20);
            }
            const unsigned m = __ballot_sync(0xffffffffu, due);
            if (due) {
                const unsigned long long ticket = base + written + __popc(m & ((1u << lane) - 1u));
                const unsigned long long slot = ticket & a.q_mask;
                volatile unsigned long long* seq = &a.q_seq[slot];
                const unsigned long long t0 = global_ns();
                bool ok = true;
                while (*seq != ticket) {  // the slot's previous item not read yet (bounded wait)
                    if (*(volatile int*)&a.ctl->abort || (long long)(global_ns() - t0) > a.barrier_timeout_ns) {
                        atomicCAS(&a.ctl->error, 0, TS_E_TIMEOUT);
                        atomicExch(&a.ctl->abort, 1);
                        ok = false;
                        break;
                    }
                    __nanosleep(64);
                }
                if (ok) {
                    __stcg(&a.q_items[slot], item);
                    __threadfence();
                    *seq = ticket + 1;
                }
            }
            written += __popc(m);
        }
        __syncwarp();
        return;
    }
}

// The queue's slots, free for their first lap.
static __global__ void flow_queue_init(unsigned long long* seq, unsigned long long n) {
    for (unsigned long long q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) seq[q] = q;
}

template <typename Real, int BX, int BY, int BZ, int WARPS, int MINB, bool VARZ_ANY, bool PENCIL, int OPT = 0>
__global__ void __launch_bounds__(WARPS * 32, MINB) flow_kernel(Args<Real> a) {
    using S = Shape<Real, BX, BY, BZ>;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int kWarpBytes = PENCIL ? PencilSmem<Real, BX>::kBytes : WarpSmem<Real, S>::kBytes;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* mine = smem + warp * kWarpBytes;
    Real* cube = reinterpret_cast<Real*>(mine);
    Real* ss = cube + S::CUBE;
    Real* mwx = ss + S::N;
    Real* mwy = mwx + 2 * S::BY * S::BZ;
    Real* mzc = mwy + 2 * S::BZ;
    uint32_t* fixedm = reinterpret_cast<uint32_t*>(mzc + kZCoef * S::BZ);
    uint32_t* dm = fixedm + S::MW;
    uint32_t* chg = dm + S::MW;
    uint32_t* chg_all = chg + S::MW;
    uint16_t* ptab = reinterpret_cast<uint16_t*>(smem + WARPS * kWarpBytes);
    int* poff = reinterpret_cast<int*>(smem + WARPS * kWarpBytes + (S::N * 2 + 15) / 16 * 16);
    uint32_t* wake = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(poff) +
                                                 ((S::NPLANES + 1) * 4 + 15) / 16 * 16);
    if (!PENCIL) {
        for (int q = threadIdx.x; q < S::N; q += blockDim.x) ptab[q] = a.plane_tab[q];
        for (int q = threadIdx.x; q <= S::NPLANES; q += blockDim.x) poff[q] = a.plane_off[q];
        for (int q = threadIdx.x; q < 12 * S::MW; q += blockDim.x) wake[q] = a.wake_mask[q];
    }
    __syncthreads();
    const int gwarp = blockIdx.x * WARPS + warp;
    const int nwarps = gridDim.x * WARPS;
    unsigned long long my_updates = 0, my_visits = 0;

    if (lane == 0) atomicCAS(&a.ctl->t_start, 0ull, global_ns());
    __syncwarp();
    // Every running field starts its launch at the first diagonal of a round.
    for (int e = gwarp; e < a.n_active; e += nwarps) {
        const int f = a.plan.field_list[e];
        if (lane == 0) a.fields[f].state->launch_rounds = 0;
        __syncwarp();
        flow_advance<Real, S::MW>(a, f, true, lane);
    }
    for (;;) {
        unsigned long long ticket = 0;
        if (lane == 0) ticket = atomicAdd(&a.ctl->q_head, 1ull);
        ticket = __shfl_sync(0xffffffffu, ticket, 0);
        const unsigned long long slot = ticket & a.q_mask;
        int state = 0;  // 1: the item is there; 2: leave
        if (lane == 0) {
            // The limit counts from the last tiles any warp queued: a long wait while others work
            // is not a failure. The poll interval grows while nothing arrives.
            unsigned long long t0 = global_ns();
            unsigned long long seen = *(volatile unsigned long long*)&a.ctl->q_tail;
            unsigned nap = 32;
            for (;;) {
                if (*(volatile unsigned long long*)&a.q_seq[slot] == ticket + 1) {
                    state = 1;
                    break;
                }
                if (*(volatile int*)&a.ctl->done || *(volatile int*)&a.ctl->abort) {
                    state = 2;
                    break;
                }
                const unsigned long long now_p = *(volatile unsigned long long*)&a.ctl->q_tail;
                if (now_p != seen) {
                    seen = now_p;
                    t0 = global_ns();
                }
                if ((long long)(global_ns() - t0) > a.barrier_timeout_ns) {
                    atomicCAS(&a.ctl->error, 0, TS_E_TIMEOUT);
                    atomicExch(&a.ctl->abort, 1);
                    state = 2;
                    break;
                }
                __nanosleep(nap);
                nap = nap < 1024 ? nap * 2 : nap;
            }
        }
        state = __shfl_sync(0xffffffffu, state, 0);
        if (state == 2) break;
        __threadfence();
        const unsigned long long e = __ldcg(&a.q_items[slot]);
        __threadfence();
        if (lane == 0) *(volatile unsigned long long*)&a.q_seq[slot] = ticket + a.q_mask + 1;  // slot free
        const int ff = int(e >> 32);
        const int sx = int(e & 1023u), sy = int((e >> 10) & 1023u), sz = int((e >> 20) & 1023u);
        const FieldDesc<Real>& fd = a.fields[ff];
        const GridDesc& g = a.grids[fd.grid];
        volatile FieldState* st = fd.state;
        const int dir = st->dir;
        const bool second = st->phase == 1;
        int ev;
        if constexpr (PENCIL) {
            // No per-ordering specialisation here: warps of one launch work on fields at different
            // orderings, and eight copies of the visit would not share the instruction cache.
            Real* halo = reinterpret_cast<Real*>(mine);
            if (VARZ_ANY && g.varz) ev = visit_pencil<Real, BX, true, false, OPT>(a, g, fd, ff, sx, sy, sz, dir, second, halo, lane);
            else ev = visit_pencil<Real, BX, false, false, OPT>(a, g, fd, ff, sx, sy, sz, dir, second, halo, lane);
        } else {
            if (VARZ_ANY && g.varz)
                ev = process_tile<Real, S, true>(a, g, fd, ff, sx, sy, sz, dir, second, cube, ss, mwx, mwy, mzc,
                                                 fixedm, dm, chg, chg_all, ptab, poff, wake, lane);
            else
                ev = process_tile<Real, S, false>(a, g, fd, ff, sx, sy, sz, dir, second, cube, ss, mwx, mwy, mzc,
                                                  fixedm, dm, chg, chg_all, ptab, poff, wake, lane);
        }
        my_updates += ev;
        my_visits += 1;
        // The last tile of the field's diagonal moves the field on.
        __threadfence();
        __syncwarp();
        int left = 0;
        if (lane == 0) left = atomicSub((int*)&st->pending, 1) - 1;
        left = __shfl_sync(0xffffffffu, left, 0);
        if (left == 0) {
            __threadfence();
            flow_advance<Real, S::MW>(a, ff, false, lane);
        }
    }
    for (int o = 16; o > 0; o >>= 1) my_updates += __shfl_down_sync(0xffffffffu, my_updates, o);
    if (lane == 0) {
        atomicAdd(&a.ctl->updates, my_updates);
        atomicAdd(&a.ctl->visits, my_visits);
    }
}

}  // namespace eik
}  // namespace ts
