// Damped LSQR on the device (Numerics/Lsqr.cs:33-152; the reference's device variant is
// Numerics/LsqrOpenCl.cs): min ‖A x − b‖² + damp² ‖x‖² by Golub–Kahan bidiagonalisation.
//
// The matrix, its transpose and every LSQR vector stay in device memory; per iteration the host
// reads back two scalars (‖u‖², ‖v‖²; ‖w‖² rides with the first) and carries the plane rotations
// and the three stopping rules exactly as the reference's loop does. Kernels: a warp per CSR row for
// A·v and Aᵀ·u, each fused with the vector update that follows it (u ← A v − α u, v ← Aᵀ u − β v) and
// with a per-block partial sum of squares; the solution update fused with w's update and its norm.
// Partial sums are reduced in a fixed order, so a solve repeats to the bit on a given device; it
// agrees with the sequential host solver to rounding (the sums are ordered differently).
//
// The transpose is the reference's (CsrMatrix.Transpose, SparseMatrix.cs:79-96): rows ascending within
// each column; built on the host for a host matrix and on the device for device-resident rows.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "host_geo.h"
#include "rays.h"

namespace ts {
namespace lsqr {

constexpr int kBlocks = 592;  // 4 blocks of 256 threads per SM; the partial-sum count
constexpr int kThreads = 256;

// y_i = (A x)_i − a · y_i for rows i (one warp per row), and the block's partial sum of y_i².
template <typename Val>
__global__ void spmv_update(int rows, const int* __restrict__ rs, const int* __restrict__ ci,
                            const Val* __restrict__ va, const double* __restrict__ x, double a,
                            double* __restrict__ y, double* __restrict__ partial) {
    __shared__ double sq[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * (kThreads / 32) + warp, nw = gridDim.x * (kThreads / 32);
    double acc2 = 0.0;
    for (int i = gw; i < rows; i += nw) {
        double s = 0.0;
        // Unrolled so that several gathers of x are in flight per lane; each lane still adds its
        // terms in order.
#pragma unroll 4
        for (int k = rs[i] + lane; k < rs[i + 1]; k += 32) s += double(va[k]) * x[ci[k]];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            const double r = s - a * y[i];
            y[i] = r;
            acc2 += r * r;
        }
    }
    if (lane == 0) sq[warp] = acc2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < kThreads / 32; q++) t += sq[q];
        partial[blockIdx.x] = t;
    }
}

// x ← x + c1·w; w ← v + c2·w; partial sums of the new w².
__global__ void update_xw(int n, const double* __restrict__ v, double c1, double c2, double* __restrict__ x,
                          double* __restrict__ w, double* __restrict__ partial) {
    __shared__ double sq[kThreads];
    double acc = 0.0;
    for (int j = blockIdx.x * kThreads + threadIdx.x; j < n; j += gridDim.x * kThreads) {
        const double wj = w[j];
        x[j] += c1 * wj;
        const double nw = v[j] + c2 * wj;
        w[j] = nw;
        acc += nw * nw;
    }
    sq[threadIdx.x] = acc;
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sq[threadIdx.x] += sq[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sq[0];
}

__global__ void scale(int n, double* __restrict__ x, double s) {
    for (int j = blockIdx.x * kThreads + threadIdx.x; j < n; j += gridDim.x * kThreads) x[j] *= s;
}

// The sum of kBlocks partials in a fixed order (one block).
__global__ void reduce_partials(const double* __restrict__ partial, int count, double* __restrict__ out) {
    __shared__ double sq[kThreads];
    double acc = 0.0;
    for (int q = threadIdx.x; q < count; q += kThreads) acc += partial[q];
    sq[threadIdx.x] = acc;
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sq[threadIdx.x] += sq[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sq[0];
}

__global__ void gather_values(int64_t nnz, const int* __restrict__ perm, const float* __restrict__ len,
                              float* __restrict__ out) {
    for (int64_t p = blockIdx.x * int64_t(kThreads) + threadIdx.x; p < nnz; p += int64_t(gridDim.x) * kThreads)
        out[p] = len[perm[p]];
}

// ---- the transpose on the device, in the reference's order -------------------------------------
// Counts per column, column pointers (a host scan of the counts), an unordered scatter, then each
// column's entries put in ascending row order by their rank among the column's rows (rows are
// distinct within a column), so the result equals CsrMatrix.Transpose entry for entry.

// Entries whose column is not below `cols` are not counted (the host then refuses the matrix).
__global__ void count_columns(int rows, int cols, const int* __restrict__ rs, const int* __restrict__ ci,
                              int* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * kThreads + threadIdx.x) >> 5; i < rows; i += (gridDim.x * kThreads) >> 5)
        for (int k = rs[i] + lane; k < rs[i + 1]; k += 32) {
            const int c = ci[k];
            if (unsigned(c) < unsigned(cols)) atomicAdd(&cnt[c], 1);
        }
}

__global__ void scatter_columns(int rows, int cols, const int* __restrict__ rs, const int* __restrict__ ci,
                                const int* __restrict__ cptr, int* __restrict__ cursor, int* __restrict__ trow,
                                int* __restrict__ tsrc) {
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * kThreads + threadIdx.x) >> 5; i < rows; i += (gridDim.x * kThreads) >> 5)
        for (int k = rs[i] + lane; k < rs[i + 1]; k += 32) {
            const int c = ci[k];
            if (unsigned(c) >= unsigned(cols)) continue;
            const int p = cptr[c] + atomicAdd(&cursor[c], 1);
            trow[p] = i;
            tsrc[p] = k;
        }
}

// One block per column: entry e goes to cptr[c] + (number of the column's rows smaller than its row).
__global__ void order_columns(int cols, const int* __restrict__ cptr, const int* __restrict__ trow,
                              const int* __restrict__ tsrc, int* __restrict__ tci, int* __restrict__ perm) {
    for (int c = blockIdx.x; c < cols; c += gridDim.x) {
        const int b = cptr[c], e = cptr[c + 1];
        for (int q = b + threadIdx.x; q < e; q += kThreads) {
            const int r = trow[q];
            int rank = 0;
            for (int t = b; t < e; t++) rank += trow[t] < r;
            tci[b + rank] = r;
            perm[b + rank] = tsrc[q];
        }
    }
}

// CsrMatrix.Transpose: column pointers, row of each transposed entry and the entry it came from.
static void transpose_host(int m, int n, const int* rs, const int* ci, std::vector<int>& trs, std::vector<int>& tci,
                           std::vector<int>& perm) {
    const int64_t nnz = rs[m];
    trs.assign(size_t(n) + 1, 0);
    for (int64_t k = 0; k < nnz; k++) trs[size_t(ci[k]) + 1]++;
    for (int c = 0; c < n; c++) trs[size_t(c) + 1] += trs[c];
    std::vector<int> next(trs.begin(), trs.end() - 1);
    tci.resize(size_t(nnz));
    perm.resize(size_t(nnz));
    for (int i = 0; i < m; i++)
        for (int k = rs[i]; k < rs[i + 1]; k++) {
            const int p = next[ci[k]]++;
            tci[p] = i;
            perm[p] = k;
        }
}

// A and its transpose on the device: values as FP64 (a host matrix), or as the float32 lengths a ray
// call leaves (widened on load: the same FP64 products, a third less traffic per non-zero).
struct System {
    int m = 0, n = 0;
    int64_t nnz = 0;
    const int *rs = nullptr, *ci = nullptr, *trs = nullptr, *tci = nullptr;
    const double *va = nullptr, *tva = nullptr;
    const float *vaf = nullptr, *tvaf = nullptr;
};

// A·x or Aᵀ·x fused with the update, on whichever value type the system holds.
static void spmv(const System& A, bool transpose, const double* x, double a, double* y, double* part,
                 cudaStream_t s) {
    const int rows = transpose ? A.n : A.m;
    const int* rs = transpose ? A.trs : A.rs;
    const int* ci = transpose ? A.tci : A.ci;
    if (A.vaf)
        spmv_update<float><<<kBlocks, kThreads, 0, s>>>(rows, rs, ci, transpose ? A.tvaf : A.vaf, x, a, y, part);
    else
        spmv_update<double><<<kBlocks, kThreads, 0, s>>>(rows, rs, ci, transpose ? A.tva : A.va, x, a, y, part);
}

// The LSQR iteration on a system already on the device (Lsqr.cs:50-150, term for term). Two reads
// per iteration: ‖u‖² (with the ‖w‖² of the previous update) and ‖v‖².
static int run(ts_ctx* ctx, const System& A, const double* b, double damp, int max_it, double atol, double btol,
               double conlim, double* x_out, ts_lsqr_info* info) {
    cudaStream_t s = ctx->stream;
    const int m = A.m, n = A.n;
    TS_BUF(ctx, u, double, "lsqr.u", std::max(1, m));
    TS_BUF(ctx, v, double, "lsqr.v", std::max(1, n));
    TS_BUF(ctx, w, double, "lsqr.w", std::max(1, n));
    TS_BUF(ctx, x, double, "lsqr.x", std::max(1, n));
    TS_BUF(ctx, part, double, "lsqr.partial", 2 * kBlocks);
    TS_BUF(ctx, scal, double, "lsqr.scalars", 4);
    double* hs = static_cast<double*>(ctx->host_buf("lsqr.host_scalars", 4 * sizeof(double)));
    if (!hs) return TS_E_NOMEM;
    auto sum_to = [&](const double* partials, int slot) {
        reduce_partials<<<1, kThreads, 0, s>>>(partials, kBlocks, scal + slot);
    };
    auto fetch = [&](int count) -> int {
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(hs, scal, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
        TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        return TS_OK;
    };
    EventPair ev;
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    cudaEventRecord(e0, s);
    auto finish = [&](int stop, int it, double bnorm, double rnorm, double acond) -> int {
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        TS_CUDA_TRY(ctx, cudaMemcpy(x_out, x, sizeof(double) * n, cudaMemcpyDeviceToHost));
        if (info) {
            info->iterations = it;
            info->stop = stop;
            info->bnorm = bnorm;
            info->rnorm = rnorm;
            info->acond = acond;
            info->device_ms = ms;
        }
        return TS_OK;
    };
    TS_CUDA_TRY(ctx, cudaMemsetAsync(x, 0, sizeof(double) * n, s));
    // β u = b (‖b‖ on the host, where b is)
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(u, b, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    double bb = 0;
    for (int i = 0; i < m; i++) bb += b[i] * b[i];
    double beta = std::sqrt(bb);
    if (beta == 0) return finish(1, 0, 0, 0, 0);
    const double bnorm = beta;
    scale<<<kBlocks, kThreads, 0, s>>>(m, u, 1.0 / beta);
    // α v = Aᵀ u (v starts at zero, so the update term vanishes)
    TS_CUDA_TRY(ctx, cudaMemsetAsync(v, 0, sizeof(double) * n, s));
    spmv(A, true, u, 0.0, v, part, s);
    sum_to(part, 1);
    if (int rc = fetch(2)) return rc;
    double alpha = std::sqrt(hs[1]);
    if (alpha == 0) return finish(2, 0, bnorm, bnorm, 0);
    scale<<<kBlocks, kThreads, 0, s>>>(n, v, 1.0 / alpha);
    // w ← v (x unchanged) with ‖w‖², read back with the first iteration's ‖u‖².
    TS_CUDA_TRY(ctx, cudaMemsetAsync(w, 0, sizeof(double) * n, s));
    update_xw<<<kBlocks, kThreads, 0, s>>>(n, v, 0.0, 0.0, x, w, part + kBlocks);
    sum_to(part + kBlocks, 2);
    double rhobar = alpha, phibar = beta;
    double ddnorm = 0, xxnorm = 0, z = 0, cs2 = -1, sn2 = 0, anorm2 = 0, damped2 = 0, rnorm = beta, acond = 0;
    const double ctol = conlim > 0 ? 1.0 / conlim : 0.0;
    int stop = 3, iterations = 0;
    for (int it = 0; it < max_it; it++) {
        iterations = it + 1;
        if (ctx->cancel_host && *ctx->cancel_host) return ctx->fail(TS_E_CANCELLED, "cancelled");
        // β u ← A v − α u
        spmv(A, false, v, alpha, u, part, s);
        sum_to(part, 0);
        if (int rc = fetch(3)) return rc;
        beta = std::sqrt(hs[0]);
        const double ww = hs[2];  // ‖w‖² of the w this iteration starts from
        if (beta > 0) {
            scale<<<kBlocks, kThreads, 0, s>>>(m, u, 1.0 / beta);
            anorm2 += alpha * alpha + beta * beta + damp * damp;
            // α v ← Aᵀ u − β v
            spmv(A, true, u, beta, v, part, s);
            sum_to(part, 1);
            if (int rc = fetch(2)) return rc;
            alpha = std::sqrt(hs[1]);
            if (alpha > 0) scale<<<kBlocks, kThreads, 0, s>>>(n, v, 1.0 / alpha);
        }
        const double rhobar1 = std::sqrt(rhobar * rhobar + damp * damp);
        const double cs1 = rhobar / rhobar1, sn1 = damp / rhobar1;
        const double psi = sn1 * phibar;
        phibar = cs1 * phibar;
        const double rho = std::sqrt(rhobar1 * rhobar1 + beta * beta);
        const double cs = rhobar1 / rho, sn = beta / rho;
        const double theta = sn * alpha;
        rhobar = -cs * alpha;
        const double phi = cs * phibar;
        phibar = sn * phibar;
        const double tau = sn * phi;
        ddnorm += ww / (rho * rho);
        // x ← x + (φ/ρ) w ; w ← v − (θ/ρ) w, and the new ‖w‖²
        update_xw<<<kBlocks, kThreads, 0, s>>>(n, v, phi / rho, -theta / rho, x, w, part + kBlocks);
        sum_to(part + kBlocks, 2);
        const double delta = sn2 * rho, gambar = -cs2 * rho, rhs = phi - delta * z;
        const double gamma = std::sqrt(gambar * gambar + theta * theta);
        cs2 = gambar / gamma;
        sn2 = theta / gamma;
        z = rhs / gamma;
        xxnorm += z * z;
        damped2 += psi * psi;
        const double anorm = std::sqrt(anorm2);
        acond = anorm * std::sqrt(ddnorm);
        const double arnorm = alpha * std::fabs(tau);
        rnorm = std::sqrt(phibar * phibar + damped2);
        const double xnorm = std::sqrt(xxnorm);
        if (ctx->lsqr_on_iteration) ctx->lsqr_on_iteration(iterations, rnorm, ctx->lsqr_user);
        const double test1 = rnorm / bnorm;
        const double test2 = arnorm / std::max(1e-300, anorm * rnorm);
        const double test3 = 1.0 / std::max(1e-300, acond);
        const double t1 = test1 / (1 + anorm * xnorm / bnorm);
        const double rtol = btol + atol * anorm * xnorm / bnorm;
        if (test1 <= rtol) { stop = 4; break; }
        if (test2 <= atol) { stop = 5; break; }
        if (ctol > 0 && test3 <= ctol) { stop = 6; break; }
        if (1 + t1 <= 1) { stop = 7; break; }
        if (1 + test2 <= 1) { stop = 8; break; }
        if (1 + test3 <= 1) { stop = 9; break; }
        if (beta == 0 || alpha == 0) { stop = 10; break; }
    }
    return finish(stop, iterations, bnorm, rnorm, acond);
}

}  // namespace lsqr
}  // namespace ts

using namespace ts::lsqr;

extern "C" {

int ts_lsqr_solve(ts_ctx* ctx, int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col, const double* val,
                  const double* b, double damp, int32_t max_iterations, double atol, double btol, double conlim,
                  double* x_out, ts_lsqr_info* info) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (info) std::memset(info, 0, sizeof(*info));
    if (m < 0 || n < 0 || (m > 0 && (!row_ptr || !b)) || (n > 0 && !x_out)) return ctx->fail(TS_E_ARG, "null array");
    if (m == 0 || n == 0) {
        if (n > 0) std::fill(x_out, x_out + n, 0.0);
        return TS_OK;
    }
    const int64_t nnz = row_ptr[m];
    if (nnz > 0 && (!col || !val)) return ctx->fail(TS_E_ARG, "null array");
    for (int64_t k = 0; k < nnz; k++)
        if (uint32_t(col[k]) >= uint32_t(n)) return ctx->fail(TS_E_ARG, "column index out of range");
    std::vector<int> trs, tci, perm;
    transpose_host(m, n, row_ptr, col, trs, tci, perm);
    std::vector<double> tva(static_cast<size_t>(nnz));
    for (int64_t p = 0; p < nnz; p++) tva[p] = val[perm[p]];
    cudaStream_t s = ctx->stream;
    TS_BUF(ctx, d_rs, int, "lsqr.rs", m + 1);
    TS_BUF(ctx, d_ci, int, "lsqr.ci", std::max<int64_t>(1, nnz));
    ctx->release("lsqr.tvaf");  // float values of earlier device rows are not needed here
    TS_BUF(ctx, d_va, double, "lsqr.va", std::max<int64_t>(1, nnz));
    TS_BUF(ctx, d_trs, int, "lsqr.trs", n + 1);
    TS_BUF(ctx, d_tci, int, "lsqr.tci", std::max<int64_t>(1, nnz));
    TS_BUF(ctx, d_tva, double, "lsqr.tva", std::max<int64_t>(1, nnz));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_rs, row_ptr, sizeof(int) * (m + 1), cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_ci, col, sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_va, val, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_trs, trs.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_tci, tci.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_tva, tva.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    System A{m, n, nnz, d_rs, d_ci, d_trs, d_tci, d_va, d_tva};
    return run(ctx, A, b, damp, max_iterations, atol, btol, conlim, x_out, info);
}

int ts_lsqr_solve_rows(ts_ctx* ctx, ts_rows* rows, int32_t n, const double* b, double damp, int32_t max_iterations,
                       double atol, double btol, double conlim, double* x_out, ts_lsqr_info* info) {
    if (!ctx || !rows) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (info) std::memset(info, 0, sizeof(*info));
    int m = 0;
    int64_t nnz = 0;
    const int *rs = nullptr, *ci = nullptr;
    const float* len = nullptr;
    ts::rays::rows_view(rows, &m, &nnz, &rs, &ci, &len);
    if (n <= 0 || m == 0 || !b || !x_out) return ctx->fail(TS_E_ARG, "empty system or null array");
    cudaStream_t s = ctx->stream;
    // The transpose built on the device in the reference's order; its values gathered there too.
    ctx->release("lsqr.va");  // FP64 values of an earlier host matrix are not needed here
    ctx->release("lsqr.tva");
    TS_BUF(ctx, d_trs, int, "lsqr.trs", n + 1);
    TS_BUF(ctx, d_tci, int, "lsqr.tci", std::max<int64_t>(1, nnz));
    TS_BUF(ctx, d_tva, float, "lsqr.tvaf", std::max<int64_t>(1, nnz));
    TS_BUF(ctx, d_perm, int, "lsqr.perm", std::max<int64_t>(1, nnz));
    TS_BUF(ctx, d_trow, int, "lsqr.trow", std::max<int64_t>(1, nnz));
    TS_BUF(ctx, d_tsrc, int, "lsqr.tsrc", std::max<int64_t>(1, nnz));
    TS_BUF(ctx, d_cnt, int, "lsqr.cnt", n);
    TS_CUDA_TRY(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(int) * n, s));
    count_columns<<<kBlocks * 8, kThreads, 0, s>>>(m, n, rs, ci, d_cnt);
    TS_CUDA_TRY(ctx, cudaGetLastError());
    std::vector<int> trs(static_cast<size_t>(n) + 1, 0);
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(trs.data() + 1, d_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    int64_t total = 0;
    for (int c = 0; c < n; c++) {
        total += trs[c + 1];
        trs[c + 1] = int(total);
    }
    if (total != nnz) return ctx->fail(TS_E_ARG, "column index beyond n");
    TS_CUDA_TRY(ctx, cudaMemcpyAsync(d_trs, trs.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
    TS_CUDA_TRY(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(int) * n, s));
    scatter_columns<<<kBlocks * 8, kThreads, 0, s>>>(m, n, rs, ci, d_trs, d_cnt, d_trow, d_tsrc);
    order_columns<<<std::min(n, 262140), kThreads, 0, s>>>(n, d_trs, d_trow, d_tsrc, d_tci, d_perm);
    gather_values<<<kBlocks * 4, kThreads, 0, s>>>(nnz, d_perm, len, d_tva);
    TS_CUDA_TRY(ctx, cudaGetLastError());
    TS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    ctx->release("lsqr.perm");
    ctx->release("lsqr.trow");
    ctx->release("lsqr.tsrc");
    ctx->release("lsqr.cnt");
    System A{m, n, nnz, rs, ci, d_trs, d_tci, nullptr, nullptr, len, d_tva};
    return run(ctx, A, b, damp, max_iterations, atol, btol, conlim, x_out, info);
}

int ts_lsqr_set_callback(ts_ctx* ctx, ts_lsqr_iteration_fn fn, void* user) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    ctx->lsqr_on_iteration = fn;
    ctx->lsqr_user = user;
    return TS_OK;
}

int ts_lsqr_selftest(ts_ctx* ctx, double* rel_err, char* msg, int32_t cap) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    // A random sparse damped system with a few non-zeros per row, as a ray matrix has
    // (LsqrOpenCl.TestSystem(3000, 1200, 12, 17), LsqrOpenCl.cs:559-573): distinct ascending columns,
    // values in [0.1, 1.1), right-hand side in [-0.5, 0.5). Its own generator (splitmix64).
    const int m = 3000, n = 1200, per_row = 12;
    uint64_t state = 17;
    auto next = [&]() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    auto uniform = [&]() { return double(next() >> 11) * (1.0 / 9007199254740992.0); };
    std::vector<int32_t> rp(m + 1, 0), ci;
    std::vector<double> va, b(m);
    for (int i = 0; i < m; i++) {
        std::vector<int32_t> c;
        while (int(c.size()) < per_row) {
            int32_t q = int32_t(next() % uint64_t(n));
            if (std::find(c.begin(), c.end(), q) == c.end()) c.push_back(q);
        }
        std::sort(c.begin(), c.end());
        for (int32_t q : c) {
            ci.push_back(q);
            va.push_back(uniform() + 0.1);
        }
        b[i] = uniform() - 0.5;
        rp[i + 1] = int32_t(ci.size());
    }
    // LsqrOpenCl.SelfTest (:541-557): damp 0.05, 300 iterations, atol = btol = 1e-12, conlim 1e10.
    std::vector<double> host(n), dev(n);
    const int host_it = ts::host::lsqr_for_selftest(m, n, rp.data(), ci.data(), va.data(), b.data(), 0.05, 300, 1e-12,
                                                    1e-12, 1e10, host.data());
    auto fn = ctx->lsqr_on_iteration;
    ctx->lsqr_on_iteration = nullptr;  // the gate reports no iterations
    ts_lsqr_info info{};
    const int rc = ts_lsqr_solve(ctx, m, n, rp.data(), ci.data(), va.data(), b.data(), 0.05, 300, 1e-12, 1e-12, 1e10,
                                 dev.data(), &info);
    ctx->lsqr_on_iteration = fn;
    char text[256];
    double rel = INFINITY;
    if (rc) {
        std::snprintf(text, sizeof text, "%s", ctx->err.c_str());
    } else {
        double worst = 0, scale = 0;
        for (int q = 0; q < n; q++) {
            worst = std::max(worst, std::fabs(dev[q] - host[q]));
            scale = std::max(scale, std::fabs(host[q]));
        }
        rel = worst / std::max(1e-300, scale);
        std::snprintf(text, sizeof text, "max |dx| %.2E of max |x| after %d iterations (host %d)", rel,
                      info.iterations, host_it);
    }
    if (rel_err) *rel_err = rel;
    if (msg && cap > 0) std::snprintf(msg, size_t(cap), "%s", text);
    if (rc) return rc;
    // LsqrOpenCl.SelfTestTolerance (:33).
    return rel <= 1e-8 ? TS_OK : ctx->fail(TS_E_SELFTEST, text);
}

}  // extern "C"
