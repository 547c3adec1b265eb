// The tiled engine's host side: lays out the job's descriptors in one device arena, seeds the
// fields, and makes the cooperative persistent launch.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "eik_engine.h"
#include "eik_engine_kernel.cuh"

namespace ts {
namespace eik {

const std::vector<TileShapeInfo>& tile_shapes() {
    // 0-3: cube tiles swept by node planes; 4-6: pencils (one lane per row of an 8×4 cross-section;
    // 6 is 4 with room for 170 registers instead of 128: 12 warps per SM and the FP64 sweep
    // orderings specialised).
    static const std::vector<TileShapeInfo> shapes = {{0, 8, 8, 8}, {1, 16, 8, 4}, {2, 8, 8, 4}, {3, 8, 4, 4},
                                                      {4, 32, 8, 4}, {5, 64, 8, 4}, {6, 32, 8, 4},
                                                      {7, 32, 8, 4}, {8, 32, 8, 4}, {9, 32, 8, 4}, {10, 32, 8, 4}};
    return shapes;
}

namespace {

// A host image of device memory: aligned sub-allocations, uploaded in one copy.
struct Arena {
    std::vector<uint8_t> h;
    size_t add(size_t bytes, size_t align = 16) {
        size_t off = (h.size() + align - 1) / align * align;
        h.resize(off + std::max<size_t>(bytes, 1), 0);
        return off;
    }
    template <typename T>
    T* at(size_t off) { return reinterpret_cast<T*>(h.data() + off); }
};

// New fields of an epoch: +inf everywhere (pads included), every tile and node due, state zero.
template <typename Real>
__global__ void init_fields_kernel(const FieldDesc<Real>* __restrict__ fields, const GridDesc* __restrict__ grids,
                                   const int* __restrict__ init_list, int mw) {
    const FieldDesc<Real>& fd = fields[init_list[blockIdx.y]];
    const GridDesc& g = grids[fd.grid];
    int64_t n = int64_t(g.pitch) * g.ny * g.nz;
    const Real inf = real_inf<Real>();
    const int64_t t0 = blockIdx.x * int64_t(blockDim.x) + threadIdx.x, stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = t0; q < n; q += stride) fd.T[q] = inf;
    int64_t nt = int64_t(g.tx) * g.ty * g.tz;
    for (int64_t q = t0; q < nt; q += stride) fd.dirty[q] = 1;
    for (int64_t q = t0; q < nt * mw; q += stride) fd.dmask[q] = 0xffffffffu;  // every node due (EikonalOpenCl.cs:411)
    if (t0 == 0) *fd.state = FieldState{};
}

template <typename Real>
__global__ void seed_fields_kernel(const FieldDesc<Real>* __restrict__ fields, const GridDesc* __restrict__ grids,
                                   const int* __restrict__ field_of, const int32_t* __restrict__ node,
                                   const double* __restrict__ t, int count) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const FieldDesc<Real>& fd = fields[field_of[q]];
    const GridDesc& g = grids[fd.grid];
    int n = node[q], i = n % g.nx, row = n / g.nx;
    fd.T[int64_t(row) * g.pitch + Layout<Real>::HX + i] = Real(t[q]);
}

// The epoch's field states, gathered for one copy to the host.
template <typename Real>
__global__ void gather_states_kernel(const FieldDesc<Real>* __restrict__ fields, int nf, FieldState* __restrict__ out) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < nf) out[f] = *fields[f].state;
}

// Padded engine fields → dense grid order of another precision (one field per blockIdx.y).
template <typename From, typename To>
__global__ void dense_convert_kernel(const From* __restrict__ a, int64_t field_stride, int pitch, int xoff, int nx,
                                     int64_t rows, To* __restrict__ b) {
    const From* src = a + blockIdx.y * field_stride;
    To* dst = b + int64_t(blockIdx.y) * rows * nx;
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < rows * nx; q += int64_t(gridDim.x) * blockDim.x) {
        int64_t r = q / nx;
        From v = src[r * pitch + xoff + (q - r * nx)];
        dst[q] = finite_r(v) ? To(v) : To(__int_as_float(0x7f800000));
    }
}

template <typename Real, int BX, int BY, int BZ, int WARPS, int MINB, bool PENCIL = false, int OPT = 0>
int launch_epoch(ts_ctx* ctx, const std::vector<const host::Grid*>& grids, const std::vector<const host::Metric*>& metrics,
                 const std::vector<EngineField*>& fl, double tol, double wake_rel, int max_rounds, ts_eik_stats* stats,
                 cudaStream_t s) {
    using S = Shape<Real, BX, BY, BZ>;
    const int nf = int(fl.size());
    const int ng = int(grids.size());
    bool any_var = false;
    for (auto* g : grids) any_var |= g->variable;

    Arena A;
    // Grids.
    std::vector<size_t> o_diag_off(ng), o_diag_tiles(ng), o_wx(ng), o_wy(ng), o_zc(ng);
    std::vector<int> tx(ng), ty(ng), tz(ng), ndiag(ng);
    size_t o_grids = A.add(sizeof(GridDesc) * ng);
    for (int gi = 0; gi < ng; gi++) {
        const host::Grid& g = *grids[gi];
        const host::Metric& m = *metrics[gi];
        tx[gi] = (g.nx + BX - 1) / BX;
        ty[gi] = (g.ny + BY - 1) / BY;
        tz[gi] = (g.nz + BZ - 1) / BZ;
        if (tx[gi] > 1024 || ty[gi] > 1024 || tz[gi] > 1024) return ctx->fail(TS_E_ARG, "grid too large for the tile table");
        ndiag[gi] = tx[gi] + ty[gi] + tz[gi] - 2;
        int nt = tx[gi] * ty[gi] * tz[gi];
        o_diag_off[gi] = A.add(sizeof(int) * (ndiag[gi] + 1));
        o_diag_tiles[gi] = A.add(sizeof(uint32_t) * nt);
        // Canonical tiles ordered by diagonal (counting sort).
        std::vector<int> cnt(ndiag[gi] + 1, 0);
        for (int c = 0; c < tz[gi]; c++)
            for (int b = 0; b < ty[gi]; b++)
                for (int a = 0; a < tx[gi]; a++) cnt[a + b + c + 1]++;
        for (int q = 0; q < ndiag[gi]; q++) cnt[q + 1] += cnt[q];
        int* doff = A.at<int>(o_diag_off[gi]);
        for (int q = 0; q <= ndiag[gi]; q++) doff[q] = cnt[q];
        std::vector<int> pos(cnt.begin(), cnt.end() - 1);
        uint32_t* dt = A.at<uint32_t>(o_diag_tiles[gi]);
        for (int c = 0; c < tz[gi]; c++)
            for (int b = 0; b < ty[gi]; b++)
                for (int a = 0; a < tx[gi]; a++) dt[pos[a + b + c]++] = uint32_t(a) | (uint32_t(b) << 10) | (uint32_t(c) << 20);
        o_wx[gi] = A.add(sizeof(Real) * m.wx.size());
        for (size_t q = 0; q < m.wx.size(); q++) A.at<Real>(o_wx[gi])[q] = Real(weight_of<Real>(m.wx[q], m.wx32[q]));
        o_wy[gi] = A.add(sizeof(Real) * m.wy.size());
        for (size_t q = 0; q < m.wy.size(); q++) A.at<Real>(o_wy[gi])[q] = Real(weight_of<Real>(m.wy[q], m.wy32[q]));
        o_zc[gi] = A.add(sizeof(Real) * std::max<size_t>(1, m.zc.size()));
        for (size_t q = 0; q < m.zc.size(); q++) A.at<Real>(o_zc[gi])[q] = Real(m.zc[q]);
    }
    // Seed tiles of each field (sorted by tile id) with their fixed-node masks; seed writes of the
    // fields this epoch initialises.
    std::vector<int> seed_begin(nf), seed_count(nf);
    std::vector<int> st_tile;
    std::vector<uint32_t> st_mask;
    std::vector<int> sc_field, init_list;
    std::vector<int32_t> sc_node;
    std::vector<double> sc_t;
    constexpr int kShape = BX | (BY << 8) | (BZ << 16);
    for (int f = 0; f < nf; f++) {
        EngineField& ef = *fl[f];
        const host::Grid& g = *grids[ef.grid];
        const int gi = ef.grid;
        if (!ef.initialized) {
            init_list.push_back(f);
            for (size_t q = 0; q < ef.seed_idx.size(); q++) {
                sc_field.push_back(f);
                sc_node.push_back(ef.seed_idx[q]);
                sc_t.push_back(ef.seed_t[q]);
            }
        }
        if (ef.seed_shape != kShape) {
            std::vector<std::pair<int, int>> tl;  // (tile, local)
            for (size_t q = 0; q < ef.seed_idx.size(); q++) {
                int node = ef.seed_idx[q];
                int i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
                int tid = ((k / BZ) * ty[gi] + j / BY) * tx[gi] + i / BX;
                int loc = ((k % BZ) * BY + j % BY) * BX + i % BX;
                tl.push_back({tid, loc});
            }
            std::sort(tl.begin(), tl.end());
            ef.seed_tiles.clear();
            ef.seed_masks.clear();
            for (size_t q = 0; q < tl.size(); q++) {
                if (q == 0 || tl[q].first != tl[q - 1].first) {
                    ef.seed_tiles.push_back(tl[q].first);
                    ef.seed_masks.resize(ef.seed_masks.size() + S::MW, 0u);
                }
                ef.seed_masks[(ef.seed_tiles.size() - 1) * S::MW + tl[q].second / 32] |= 1u << (tl[q].second % 32);
            }
            ef.seed_shape = kShape;
        }
        seed_begin[f] = int(st_tile.size());
        st_tile.insert(st_tile.end(), ef.seed_tiles.begin(), ef.seed_tiles.end());
        st_mask.insert(st_mask.end(), ef.seed_masks.begin(), ef.seed_masks.end());
        seed_count[f] = int(ef.seed_tiles.size());
    }
    size_t o_seed_tile = A.add(sizeof(int) * std::max<size_t>(1, st_tile.size()));
    std::copy(st_tile.begin(), st_tile.end(), A.at<int>(o_seed_tile));
    size_t o_seed_mask = A.add(sizeof(uint32_t) * std::max<size_t>(1, st_mask.size()));
    std::copy(st_mask.begin(), st_mask.end(), A.at<uint32_t>(o_seed_mask));
    size_t o_sc_field = A.add(sizeof(int) * sc_field.size());
    std::copy(sc_field.begin(), sc_field.end(), A.at<int>(o_sc_field));
    size_t o_sc_node = A.add(sizeof(int32_t) * sc_node.size());
    std::copy(sc_node.begin(), sc_node.end(), A.at<int32_t>(o_sc_node));
    size_t o_sc_t = A.add(sizeof(double) * sc_t.size(), 8);
    std::copy(sc_t.begin(), sc_t.end(), A.at<double>(o_sc_t));
    size_t o_init = A.add(sizeof(int) * init_list.size());
    std::copy(init_list.begin(), init_list.end(), A.at<int>(o_init));
    // Node planes of the canonical tile.
    size_t o_ptab = A.add(sizeof(uint16_t) * S::N);
    size_t o_poff = A.add(sizeof(int) * (S::NPLANES + 1));
    if (!PENCIL) {  // cube tiles only: a pencil needs no plane table
        std::vector<int> cnt(S::NPLANES + 1, 0);
        for (int k = 0; k < BZ; k++)
            for (int j = 0; j < BY; j++)
                for (int i = 0; i < BX; i++) cnt[i + j + k + 1]++;
        for (int p = 0; p < S::NPLANES; p++) cnt[p + 1] += cnt[p];
        std::copy(cnt.begin(), cnt.end(), A.at<int>(o_poff));
        std::vector<int> pos(cnt.begin(), cnt.end() - 1);
        uint16_t* pt = A.at<uint16_t>(o_ptab);
        for (int k = 0; k < BZ; k++)
            for (int j = 0; j < BY; j++)
                for (int i = 0; i < BX; i++) pt[pos[i + j + k]++] = uint16_t(i | (j << 5) | (k << 10));
    }
    // Wake masks: for each stencil offset, the tile nodes a changed node at that offset reaches
    // without leaving its row, column or plane.
    size_t o_wake = A.add(sizeof(uint32_t) * 12 * S::MW);
    if (!PENCIL) {
        uint32_t* wm = A.at<uint32_t>(o_wake);
        for (int d = 0; d < 12; d++) {
            int axis = d >> 2, r = d & 3;
            int delta = ((r & 1) ? -1 : 1) * ((r & 2) ? 2 : 1);
            int B = axis == 0 ? BX : axis == 1 ? BY : BZ;
            for (int L = 0; L < S::N; L++) {
                int pos = axis == 0 ? L % BX : axis == 1 ? (L / BX) % BY : L / (BX * BY);
                int src = pos - delta;
                if (src >= 0 && src < B) wm[d * S::MW + L / 32] |= 1u << (L % 32);
            }
        }
    }
    // Plan: one group per grid with running fields, fields ordered by group.
    std::vector<int> group_grid, group_first, field_list;
    std::vector<int> group_nf;
    int running = 0;
    for (int gi = 0; gi < ng; gi++) {
        int first = int(field_list.size());
        for (int f = 0; f < nf; f++)
            if (fl[f]->grid == gi && fl[f]->status == 0) field_list.push_back(f);
        if (int(field_list.size()) > first) {
            group_grid.push_back(gi);
            group_first.push_back(first);
            group_nf.push_back(int(field_list.size()) - first);
        }
    }
    running = int(field_list.size());
    const int G = int(group_grid.size());
    int maxdiag = 0;
    for (int gg = 0; gg < G; gg++) maxdiag = std::max(maxdiag, ndiag[group_grid[gg]]);
    size_t o_group_grid = A.add(sizeof(int) * std::max(1, G));
    std::copy(group_grid.begin(), group_grid.end(), A.at<int>(o_group_grid));
    size_t o_group_first = A.add(sizeof(int) * std::max(1, G));
    std::copy(group_first.begin(), group_first.end(), A.at<int>(o_group_first));
    size_t o_field_list = A.add(sizeof(int) * std::max<size_t>(1, field_list.size()));
    std::copy(field_list.begin(), field_list.end(), A.at<int>(o_field_list));
    size_t o_pre = A.add(sizeof(int) * size_t(std::max(1, maxdiag)) * (G + 1));
    int max_items = 0;
    for (int q = 0; q < maxdiag; q++) {
        int* pre = A.at<int>(o_pre) + size_t(q) * (G + 1);
        int64_t acc = 0;
        for (int gg = 0; gg < G; gg++) {
            pre[gg] = int(acc);
            int gi = group_grid[gg];
            int cnt = 0;
            if (q < ndiag[gi]) cnt = A.at<int>(o_diag_off[gi])[q + 1] - A.at<int>(o_diag_off[gi])[q];
            acc += int64_t(group_nf[gg]) * cnt;
        }
        if (acc > INT32_MAX / 2) return ctx->fail(TS_E_ARG, "too many tiles in one diagonal step");
        pre[G] = int(acc);
        max_items = std::max(max_items, int(acc));
    }
    // Flow scheduler queue: room for twice the tiles all fields can have outstanding at once (each
    // field has one diagonal in flight).
    size_t qcap = 1024;
    if (ctx->scheduler == 1) {
        size_t need = 0;
        for (int f = 0; f < nf; f++) {
            const int gi = fl[f]->grid;
            const int* doff = A.at<int>(o_diag_off[gi]);
            int mx = 0;
            for (int q = 0; q < ndiag[gi]; q++) mx = std::max(mx, doff[q + 1] - doff[q]);
            need += size_t(mx);
        }
        while (qcap < 2 * need) qcap *= 2;
    }
    // Fields, control, state copies.
    size_t o_fields = A.add(sizeof(FieldDesc<Real>) * nf);
    size_t o_ctl = A.add(sizeof(Control));
    size_t o_states = A.add(sizeof(FieldState) * nf);

    uint8_t* D = static_cast<uint8_t*>(ctx->buf("eng.arena", A.h.size()));
    if (!D) return TS_E_NOMEM;
    auto* worklist = static_cast<unsigned long long*>(ctx->buf("eng.worklist", 16 * size_t(std::max(1, max_items))));
    if (!worklist) return TS_E_NOMEM;
    const bool flow = ctx->scheduler == 1;
    unsigned long long* q_items = nullptr;
    unsigned long long* q_seq = nullptr;
    if (flow) {
        q_items = static_cast<unsigned long long*>(ctx->buf("eng.q_items", 8 * qcap));
        q_seq = static_cast<unsigned long long*>(ctx->buf("eng.q_seq", 8 * qcap));
        if (!q_items || !q_seq) return TS_E_NOMEM;
    }
    for (int gi = 0; gi < ng; gi++) {
        GridDesc gd{};
        const host::Grid& g = *grids[gi];
        gd.nx = g.nx; gd.ny = g.ny; gd.nz = g.nz;
        gd.tx = tx[gi]; gd.ty = ty[gi]; gd.tz = tz[gi];
        gd.ndiag = ndiag[gi];
        gd.varz = g.variable ? 1 : 0;
        gd.diag_off = reinterpret_cast<const int*>(D + o_diag_off[gi]);
        gd.diag_tiles = reinterpret_cast<const uint32_t*>(D + o_diag_tiles[gi]);
        gd.wx = D + o_wx[gi];
        gd.wy = D + o_wy[gi];
        gd.zc = D + o_zc[gi];
        gd.wz1 = weight_of<Real>(metrics[gi]->wz1, metrics[gi]->wz1_32);
        gd.wz2 = weight_of<Real>(metrics[gi]->wz2, metrics[gi]->wz2_32);
        gd.pitch = Layout<Real>::pitch(tx[gi], BX);
        A.at<GridDesc>(o_grids)[gi] = gd;
    }
    for (int f = 0; f < nf; f++) {
        const EngineField& ef = *fl[f];
        FieldDesc<Real> fd{};
        fd.T = static_cast<Real*>(ef.T);
        fd.s = static_cast<const Real*>(ef.slowness);
        fd.dirty = ef.dirty;
        fd.dmask = ef.dmask;
        fd.grid = ef.grid;
        fd.seed_begin = seed_begin[f];
        fd.seed_count = seed_count[f];
        fd.cap = ef.cap;
        fd.seed_tile_lo = seed_count[f] ? st_tile[seed_begin[f]] : 1;
        fd.seed_tile_hi = seed_count[f] ? st_tile[seed_begin[f] + seed_count[f] - 1] : 0;
        fd.state = static_cast<FieldState*>(ef.state);
        A.at<FieldDesc<Real>>(o_fields)[f] = fd;
    }
    A.at<Control>(o_ctl)->running = running;

    // The work of the epoch, enqueued on stream s: arena upload (from a pinned image), new fields'
    // initialisation and seeds, the engine launch, and the control block and field states back to
    // pinned host memory. Recorded directly, or captured once into a CUDA graph and replayed while
    // the same job (same arena bytes, same buffers) is solved again.
    uint8_t* image = static_cast<uint8_t*>(ctx->host_buf("eng.arena.image", A.h.size()));
    Control* ctl_h = static_cast<Control*>(ctx->host_buf("eng.ctl", sizeof(Control)));
    FieldState* st_h = static_cast<FieldState*>(ctx->host_buf("eng.states", sizeof(FieldState) * std::max(1, nf)));
    if (!image || !ctl_h || !st_h) return TS_E_NOMEM;
    std::memcpy(image, A.h.data(), A.h.size());
    *ctl_h = Control{};

    Args<Real> args{};
    args.grids = reinterpret_cast<const GridDesc*>(D + o_grids);
    args.fields = reinterpret_cast<const FieldDesc<Real>*>(D + o_fields);
    args.seed_tile = reinterpret_cast<const int*>(D + o_seed_tile);
    args.seed_mask = reinterpret_cast<const uint32_t*>(D + o_seed_mask);
    args.plane_tab = reinterpret_cast<const uint16_t*>(D + o_ptab);
    args.plane_off = reinterpret_cast<const int*>(D + o_poff);
    args.wake_mask = reinterpret_cast<const uint32_t*>(D + o_wake);
    args.ctl = reinterpret_cast<Control*>(D + o_ctl);
    args.cancel = ctx->cancel_dev;
    args.plan.ngroups = G;
    args.plan.maxdiag = maxdiag;
    args.plan.group_grid = reinterpret_cast<const int*>(D + o_group_grid);
    args.plan.group_first = reinterpret_cast<const int*>(D + o_group_first);
    args.plan.field_list = reinterpret_cast<const int*>(D + o_field_list);
    args.plan.pre = reinterpret_cast<const int*>(D + o_pre);
    args.n_active = int(field_list.size());
    args.worklist = worklist;
    args.worklist_cap = std::max(1, max_items);
    args.max_rounds_per_launch = max_rounds;
    args.epoch_budget_ns = (flow && max_rounds > 0) ? (long long)(ctx->epoch_budget_ms * 1e6) : 0;
    args.barrier_timeout_ns = 5000000000LL;
    args.q_items = q_items;
    args.q_seq = q_seq;
    args.q_mask = qcap - 1;
    args.tol = Real(tol);
    args.wake_rel = Real(wake_rel);
    args.causal = wake_rel > 0 ? 1 : 0;  // fast mode: threshold and causal wakes together
    const int smem = PENCIL ? WARPS * PencilSmem<Real, BX>::kBytes : engine_smem_bytes<Real, S>(WARPS);
    void* kfn = flow ? (any_var ? (void*)flow_kernel<Real, BX, BY, BZ, WARPS, MINB, true, PENCIL, OPT>
                               : (void*)flow_kernel<Real, BX, BY, BZ, WARPS, MINB, false, PENCIL, OPT>)
                     : (any_var ? (void*)engine_kernel<Real, BX, BY, BZ, WARPS, MINB, true, PENCIL, OPT>
                                : (void*)engine_kernel<Real, BX, BY, BZ, WARPS, MINB, false, PENCIL, OPT>);
    TS_CUDA_TRY(ctx, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    TS_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, WARPS * 32, smem));
    if (per_sm < 1) return ctx->fail(TS_E_CUDA, "engine kernel does not fit on an SM");
    const int blocks = per_sm * ctx->sm_count;
    void* params[] = {&args};
    int64_t maxn = 0;
    for (int f : init_list) {
        const host::Grid& g = *grids[fl[f]->grid];
        maxn = std::max(maxn, int64_t(Layout<Real>::pitch(tx[fl[f]->grid], BX)) * g.ny * g.nz);
    }
    cudaEvent_t k0 = nullptr, k1 = nullptr;
    auto enqueue = [&](bool timed) -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(D, image, A.h.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        for (size_t c0 = 0; c0 < init_list.size(); c0 += 65535) {
            unsigned cnt = unsigned(std::min<size_t>(65535, init_list.size() - c0));
            dim3 grid(unsigned(std::min<int64_t>((maxn + 255) / 256, 512)), cnt);
            init_fields_kernel<Real><<<grid, 256, 0, s>>>(reinterpret_cast<const FieldDesc<Real>*>(D + o_fields),
                                                          reinterpret_cast<const GridDesc*>(D + o_grids),
                                                          reinterpret_cast<const int*>(D + o_init) + c0, S::MW);
        }
        int cnt = int(sc_node.size());
        if (cnt > 0)
            seed_fields_kernel<Real><<<(cnt + 255) / 256, 256, 0, s>>>(
                reinterpret_cast<const FieldDesc<Real>*>(D + o_fields), reinterpret_cast<const GridDesc*>(D + o_grids),
                reinterpret_cast<const int*>(D + o_sc_field), reinterpret_cast<const int32_t*>(D + o_sc_node),
                reinterpret_cast<const double*>(D + o_sc_t), cnt);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (running > 0 && flow) {
            flow_queue_init<<<int(std::min<size_t>((qcap + 255) / 256, 1024)), 256, 0, s>>>(q_seq, qcap);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (running > 0) {
            if (timed) cudaEventRecord(k0, s);
            e = cudaLaunchCooperativeKernel(kfn, dim3(blocks), dim3(WARPS * 32), params, smem, s);
            if (timed) cudaEventRecord(k1, s);
            if (e != cudaSuccess) return e;
        }
        gather_states_kernel<Real><<<(nf + 127) / 128, 128, 0, s>>>(reinterpret_cast<const FieldDesc<Real>*>(D + o_fields),
                                                                    nf, reinterpret_cast<FieldState*>(D + o_states));
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(ctl_h, D + o_ctl, sizeof(Control), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
        return cudaMemcpyAsync(st_h, D + o_states, sizeof(FieldState) * nf, cudaMemcpyDeviceToHost, s);
    };
    bool graphed = false;
    if (ctx->use_graph && max_rounds <= 0) {
        // The job's signature: its arena bytes and the device buffers the work touches.
        unsigned long long sig = 1469598103934665603ULL;
        auto mix = [&](const void* p, size_t n) {
            const uint8_t* b = static_cast<const uint8_t*>(p);
            for (size_t q = 0; q < n; q++) sig = (sig ^ b[q]) * 1099511628211ULL;
        };
        mix(A.h.data(), A.h.size());
        uintptr_t ptrs[4] = {uintptr_t(D), uintptr_t(worklist), uintptr_t(image), uintptr_t(kfn)};
        mix(ptrs, sizeof ptrs);
        if (ctx->graph_exec && ctx->graph_sig == sig) {
            TS_CUDA_TRY(ctx, cudaGraphLaunch(ctx->graph_exec, s));
            ctx->graph_replays++;
            graphed = true;
        } else {
            ctx->drop_graph();
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t we = enqueue(false);
                e = cudaStreamEndCapture(s, &graph);
                if (we != cudaSuccess) e = we;
            }
            if (e == cudaSuccess && graph) e = cudaGraphInstantiate(&ctx->graph_exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e == cudaSuccess && ctx->graph_exec) {
                ctx->graph_sig = sig;
                TS_CUDA_TRY(ctx, cudaGraphLaunch(ctx->graph_exec, s));
                graphed = true;
            } else {
                cudaGetLastError();  // capture unsupported here: run the work directly
                ctx->drop_graph();
            }
        }
    }
    if (!graphed) {
        cudaEventCreate(&k0);
        cudaEventCreate(&k1);
        cudaError_t e = enqueue(true);
        if (e != cudaSuccess) {
            cudaEventDestroy(k0);
            cudaEventDestroy(k1);
            TS_CUDA_TRY(ctx, e);
        }
    }
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    for (int f : init_list) fl[f]->initialized = true;
    const Control ctl = *ctl_h;
    float kms = 0;
    if (!graphed && running > 0) cudaEventElapsedTime(&kms, k0, k1);
    if (k0) cudaEventDestroy(k0);
    if (k1) cudaEventDestroy(k1);
    if (stats) {
        stats->kernel_ms += kms;
        stats->node_updates += int64_t(ctl.updates);
        stats->tile_visits += int64_t(ctl.visits);
        stats->launches += running > 0 ? 1 : 0;
    }
    std::vector<FieldState> st(st_h, st_h + nf);
    for (int f = 0; f < nf; f++) {
        fl[f]->status = st[f].status;
        fl[f]->rounds[0] = st[f].rounds0;
        fl[f]->rounds[1] = st[f].rounds1;
    }
    if (ctl.error == TS_E_CANCELLED) return ctx->fail(TS_E_CANCELLED, "cancelled");
    if (ctl.error) return ctx->fail(ctl.error, "engine: a device-side wait ran out (barrier timeout)");
    return TS_OK;
}

}  // namespace

// Fields of the job in dense grid order: same precision → strided copies; otherwise converted on the
// device in blocks of fields, then copied.
int fields_to_dense_host(ts_ctx* ctx, const EngineJob& job, int precision, void* out, int out_type) {
    const size_t rsz = 8;  // a double, or the FP32 precision's float pair
    const size_t osz = out_type == TS_OUT_F64 ? 8 : 4;
    const bool same = precision == TS_PRECISION_F64 && out_type == TS_OUT_F64;
    char* dst = static_cast<char*>(out);
    for (size_t f = 0; f < job.fields.size(); f++) {
        const host::Grid& g = *job.grids[job.fields[f].grid];
        const int pitch = job.pitch[job.fields[f].grid];
        const int64_t rows = int64_t(g.ny) * g.nz, n = rows * g.nx;
        const char* src = static_cast<const char*>(job.fields[f].T);
        if (same) {
            TS_CUDA_TRY(ctx, cudaMemcpy2DAsync(dst, g.nx * osz, src + job.xoff * rsz, pitch * rsz, g.nx * rsz, rows,
                                               cudaMemcpyDeviceToHost, ctx->stream));
        } else {
            void* stage = ctx->buf("out.stage", size_t(n) * osz);
            if (!stage) return TS_E_NOMEM;
            int blocks = int(std::min<int64_t>((n + 255) / 256, 4096));
            if (precision == TS_PRECISION_F64)
                dense_convert_kernel<double, float><<<dim3(blocks, 1), 256, 0, ctx->stream>>>(
                    reinterpret_cast<const double*>(src), 0, pitch, job.xoff, g.nx, rows, static_cast<float*>(stage));
            else if (osz == 8)
                dense_convert_kernel<Pair, double><<<dim3(blocks, 1), 256, 0, ctx->stream>>>(
                    reinterpret_cast<const Pair*>(src), 0, pitch, job.xoff, g.nx, rows, static_cast<double*>(stage));
            else
                dense_convert_kernel<Pair, float><<<dim3(blocks, 1), 256, 0, ctx->stream>>>(
                    reinterpret_cast<const Pair*>(src), 0, pitch, job.xoff, g.nx, rows, static_cast<float*>(stage));
            TS_CUDA_TRY(ctx, cudaGetLastError());
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(dst, stage, size_t(n) * osz, cudaMemcpyDeviceToHost, ctx->stream));
            TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        }
        dst += size_t(n) * osz;
    }
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return TS_OK;
}

// One field as a dense float32 table on the device (the .qttb rounding).
int field_to_dense_f32_device(ts_ctx* ctx, const host::Grid& g, const FieldLayout& L, const void* T, int precision,
                              float* out, cudaStream_t s) {
    const int64_t rows = int64_t(g.ny) * g.nz, n = rows * g.nx;
    int blocks = int(std::min<int64_t>((n + 255) / 256, 2048));
    if (precision == TS_PRECISION_F64)
        dense_convert_kernel<double, float><<<dim3(blocks, 1), 256, 0, s>>>(static_cast<const double*>(T), 0, L.pitch,
                                                                            L.xoff, g.nx, rows, out);
    else
        dense_convert_kernel<Pair, float><<<dim3(blocks, 1), 256, 0, s>>>(static_cast<const Pair*>(T), 0, L.pitch,
                                                                          L.xoff, g.nx, rows, out);
    TS_CUDA_TRY(ctx, cudaGetLastError());
    return TS_OK;
}

// Fields of a job as dense float32 tables on the device, one after another.
int fields_to_dense_f32_device(ts_ctx* ctx, const EngineJob& job, int precision, float* out) {
    for (const auto& f : job.fields) {
        const host::Grid& g = *job.grids[f.grid];
        FieldLayout L = field_layout(g, job.tile, precision);
        int rc = field_to_dense_f32_device(ctx, g, L, f.T, precision, out, ctx->stream);
        if (rc) return rc;
        out += g.count();
    }
    return TS_OK;
}

template <typename Real>
int engine_epoch(ts_ctx* ctx, const std::vector<const host::Grid*>& grids,
                 const std::vector<const host::Metric*>& metrics, const std::vector<EngineField*>& fields,
                 double tol, double wake_rel, int tile, int max_rounds, ts_eik_stats* stats, cudaStream_t s) {
    if (fields.empty()) return TS_OK;
    // Warps per block sized so that two or three blocks fill an SM's shared memory.
    constexpr bool F64 = sizeof(Real) == 8;  // 8-byte values: shared memory as FP64 (Pair too)
    switch (tile) {
        case 1: return launch_epoch<Real, 16, 8, 4, F64 ? 5 : 8, 2>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        case 2: return launch_epoch<Real, 8, 8, 4, F64 ? 6 : 8, F64 ? 3 : 2>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        case 3: return launch_epoch<Real, 8, 4, 4, 8, 3>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        case 4: return launch_epoch<Real, 32, 8, 4, 4, 4, true>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        case 5: return launch_epoch<Real, 64, 8, 4, 4, F64 ? 2 : 4, true>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        case 6: return launch_epoch<Real, 32, 8, 4, 4, F64 ? 3 : 4, true>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        // 7, 8: 32-wide pencils at 16 warps per SM (128 registers), two-deep prefetch, weights read
        // where used; 8 with the sweep ordering fixed at compile time.
        case 7: return launch_epoch<Real, 32, 8, 4, 4, 4, true, kRing2 | kLazyW>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        case 8: return launch_epoch<Real, 32, 8, 4, 4, 4, true, kRing2 | kLazyW | kSpecAll>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        // 9: as 8 with the neighbour values fetched again for the wake tests (fewer live registers);
        // 10: as 6 (12 warps per SM) with the same register savings.
        case 9: return launch_epoch<Real, 32, 8, 4, 4, 4, true, kRing2 | kLazyW | kSpecAll | kReshuffle>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        case 10: return launch_epoch<Real, 32, 8, 4, 4, F64 ? 3 : 4, true, kRing2 | kLazyW | kReshuffle>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
        default: return launch_epoch<Real, 8, 8, 8, F64 ? 5 : 8, 1>(ctx, grids, metrics, fields, tol, wake_rel, max_rounds, stats, s);
    }
}

FieldLayout field_layout(const host::Grid& g, int tile, int precision) {
    int bx = 8, by = 8, bz = 8;
    for (const auto& t : tile_shapes())
        if (t.id == tile) { bx = t.bx; by = t.by; bz = t.bz; }
    const int hx = 2;  // 16 bytes of 8-byte values (a double, or the FP32 precision's float pair)
    (void)precision;
    const int tx = (g.nx + bx - 1) / bx, ty = (g.ny + by - 1) / by, tz = (g.nz + bz - 1) / bz;
    FieldLayout L;
    L.pitch = hx + tx * bx + hx;
    L.xoff = hx;
    L.tiles = tx * ty * tz;
    L.mask_words = L.tiles * ((bx * by * bz + 31) / 32);
    L.rows_ = int64_t(g.ny) * g.nz;
    return L;
}

int64_t FieldLayout::elems() const { return int64_t(pitch) * rows_; }

static size_t up256(size_t b) { return (b + 255) / 256 * 256; }

int64_t FieldLayout::bytes(int precision) const {
    const size_t esz = 8;
    (void)precision;
    return int64_t(up256(size_t(elems()) * esz) + up256(size_t(tiles)) + up256(4 * size_t(mask_words)) + 256);
}

void engine_field_place(EngineField& f, const FieldLayout& L, int precision, void* block) {
    const size_t esz = 8;
    (void)precision;
    char* p = static_cast<char*>(block);
    f.T = p;
    p += up256(size_t(L.elems()) * esz);
    f.dirty = reinterpret_cast<uint8_t*>(p);
    p += up256(size_t(L.tiles));
    f.dmask = reinterpret_cast<uint32_t*>(p);
    p += up256(4 * size_t(L.mask_words));
    f.state = p;
}

template <typename Real>
int engine_run(ts_ctx* ctx, EngineJob& job, ts_eik_stats* stats) {
    if (job.fields.empty()) return TS_OK;
    const int precision = precision_of<Real>();
    // Every field's buffers from one pooled block of the context.
    std::vector<FieldLayout> layouts;
    for (auto* g : job.grids) layouts.push_back(field_layout(*g, job.tile, precision));
    size_t total = 0;
    for (auto& f : job.fields) total += size_t(layouts[f.grid].bytes(precision));
    char* pool = static_cast<char*>(ctx->buf("eng.fields", total));
    if (!pool) return TS_E_NOMEM;
    std::vector<EngineField*> fl;
    for (auto& f : job.fields) {
        engine_field_place(f, layouts[f.grid], precision, pool);
        pool += layouts[f.grid].bytes(precision);
        f.initialized = false;
        f.status = 0;
        fl.push_back(&f);
    }
    job.pitch.clear();
    for (auto& L : layouts) job.pitch.push_back(L.pitch);
    job.xoff = layouts.empty() ? 0 : layouts[0].xoff;
    return engine_epoch<Real>(ctx, job.grids, job.metrics, fl, job.tol, job.wake_rel, job.tile, 0, stats, ctx->stream);
}

// Fields [f0, f1) of a job (after engine_run) converted to dense grid order of out_type into dst, on s.
template <typename Real>
static int fields_to_dense_device(ts_ctx* ctx, const EngineJob& job, size_t f0, size_t f1, void* dst, int out_type,
                                  cudaStream_t s) {
    char* d = static_cast<char*>(dst);
    const size_t osz = out_type == TS_OUT_F64 ? 8 : 4;
    for (size_t f = f0; f < f1; f++) {
        const host::Grid& g = *job.grids[job.fields[f].grid];
        const int pitch = job.pitch[job.fields[f].grid];
        const int64_t rows = int64_t(g.ny) * g.nz, n = rows * g.nx;
        const int blocks = int(std::min<int64_t>((n + 255) / 256, 4096));
        const Real* src = static_cast<const Real*>(job.fields[f].T);
        if (osz == 8)
            dense_convert_kernel<Real, double><<<dim3(blocks, 1), 256, 0, s>>>(src, 0, pitch, job.xoff, g.nx, rows,
                                                                               reinterpret_cast<double*>(d));
        else
            dense_convert_kernel<Real, float><<<dim3(blocks, 1), 256, 0, s>>>(src, 0, pitch, job.xoff, g.nx, rows,
                                                                              reinterpret_cast<float*>(d));
        TS_CUDA_TRY(ctx, cudaGetLastError());
        d += size_t(n) * osz;
    }
    return TS_OK;
}

template <typename Real>
int engine_run_to_host(ts_ctx* ctx, EngineJob& job, void* out, int out_type, ts_eik_stats* stats) {
    const size_t nf = job.fields.size(), half = (nf + 1) / 2;
    const size_t osz = out_type == TS_OUT_F64 ? 8 : 4;
    if (!ctx->copy_stream) TS_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    size_t bytes[2] = {0, 0};
    for (size_t f = 0; f < nf; f++) bytes[f < half ? 0 : 1] += size_t(job.grids[job.fields[f].grid]->count()) * osz;
    void* stage = ctx->buf("out.pipeline", std::max(bytes[0], bytes[1]));
    if (!stage) return TS_E_NOMEM;
    EventPair converted, copied;
    char* dst = static_cast<char*>(out);
    int rc = TS_OK;
    for (int part = 0; part < 2 && rc == TS_OK; part++) {
        const size_t f0 = part == 0 ? 0 : half, f1 = part == 0 ? half : nf;
        if (f0 == f1) continue;
        // The part as a job of its own (its fields move in and back out).
        EngineJob sub;
        sub.grids = job.grids;
        sub.metrics = job.metrics;
        sub.tol = job.tol;
        sub.wake_rel = job.wake_rel;
        sub.tile = job.tile;
        for (size_t f = f0; f < f1; f++) sub.fields.push_back(std::move(job.fields[f]));
        rc = engine_run<Real>(ctx, sub, stats);
        if (rc == TS_OK) {
            // The stage is free once the previous part's copy has read it.
            if (part == 1) TS_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, copied.a, 0));
            rc = fields_to_dense_device<Real>(ctx, sub, 0, sub.fields.size(), stage, out_type, ctx->stream);
        }
        if (rc == TS_OK) {
            TS_CUDA_TRY(ctx, cudaEventRecord(converted.a, ctx->stream));
            TS_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy_stream, converted.a, 0));
            TS_CUDA_TRY(ctx, cudaMemcpyAsync(dst, stage, bytes[part], cudaMemcpyDeviceToHost, ctx->copy_stream));
            TS_CUDA_TRY(ctx, cudaEventRecord(copied.a, ctx->copy_stream));
            dst += bytes[part];
        }
        job.pitch = sub.pitch;
        job.xoff = sub.xoff;
        for (size_t f = f0; f < f1; f++) job.fields[f] = std::move(sub.fields[f - f0]);
    }
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->copy_stream));
    return rc;
}

template int engine_run<Pair>(ts_ctx*, EngineJob&, ts_eik_stats*);
template int engine_run_to_host<double>(ts_ctx*, EngineJob&, void*, int, ts_eik_stats*);
template int engine_run_to_host<Pair>(ts_ctx*, EngineJob&, void*, int, ts_eik_stats*);
template int engine_run<double>(ts_ctx*, EngineJob&, ts_eik_stats*);
template int engine_epoch<Pair>(ts_ctx*, const std::vector<const host::Grid*>&, const std::vector<const host::Metric*>&,
                                 const std::vector<EngineField*>&, double, double, int, int, ts_eik_stats*, cudaStream_t);
template int engine_epoch<double>(ts_ctx*, const std::vector<const host::Grid*>&, const std::vector<const host::Metric*>&,
                                  const std::vector<EngineField*>&, double, double, int, int, ts_eik_stats*, cudaStream_t);

}  // namespace eik
}  // namespace ts
