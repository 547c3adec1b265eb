// The reference's device LSQR kernels (LsqrOpenCl.cs) run on the CPU from their own text — TEST
// INFRASTRUCTURE ONLY.
//
// `Source` (FP64) and `PairedSource` (float pairs hi + lo) of
// src/TomoStar.Core/Numerics/LsqrOpenCl.cs:41-176, extracted into oracle/_ref/lsqr_fp64.cl and
// oracle/_ref/lsqr_paired.cl by oracle/ref_extract.py. Each export is one launch as LsqrOpenCl.Launch
// makes it (LsqrOpenCl.cs:428-433: global size rounded up to GroupSize = 256), run as a loop over the
// work items. dot_partial (a work-group reduction with barriers) is not driven here.
#include "ref_shim.h"

thread_local RefItem ref_item;

namespace lsqr64 {
#include "lsqr_fp64.cl"
}
namespace lsqr32 {
#include "lsqr_paired.cl"
}

namespace {
constexpr size_t kGroupSize = 256;  // LsqrOpenCl.GroupSize

template <typename F>
void launch(int n, F&& body) {
    const size_t global = ((size_t)n + kGroupSize - 1) / kGroupSize * kGroupSize;
    for (size_t q = 0; q < global; q++) {
        ref_item.gid[0] = q;
        body();
    }
}

float2* pairs(float* p) { return reinterpret_cast<float2*>(p); }
const float2* pairs(const float* p) { return reinterpret_cast<const float2*>(p); }
float2 pair(const float* p) { return make_float2(p[0], p[1]); }
}  // namespace

extern "C" {

void ref_spmv_f64(int rows, const int* rs, const int* ci, const double* va, const double* x, double* y) {
    launch(rows, [&] { lsqr64::spmv(rows, rs, ci, va, x, y); });
}
void ref_xmby_f64(int n, const double* x, double b, double* y) {
    launch(n, [&] { lsqr64::xmby(n, x, b, y); });
}
void ref_xpby_f64(int n, const double* x, double b, double* y) {
    launch(n, [&] { lsqr64::xpby(n, x, b, y); });
}
void ref_axpy_f64(int n, double a, const double* x, double* y) {
    launch(n, [&] { lsqr64::axpy(n, a, x, y); });
}
void ref_scal_f64(int n, double* x, double s) {
    launch(n, [&] { lsqr64::scal(n, x, s); });
}

// Paired forms: every value is two floats (hi, lo), arrays of 2·len floats.
void ref_spmv_paired(int rows, const int* rs, const int* ci, const float* va, const float* x, float* y) {
    launch(rows, [&] { lsqr32::spmv(rows, rs, ci, pairs(va), pairs(x), pairs(y)); });
}
void ref_xmby_paired(int n, const float* x, const float* b, float* y) {
    launch(n, [&] { lsqr32::xmby(n, pairs(x), pair(b), pairs(y)); });
}
void ref_axpy_paired(int n, const float* a, const float* x, float* y) {
    launch(n, [&] { lsqr32::axpy(n, pair(a), pairs(x), pairs(y)); });
}
void ref_scal_paired(int n, float* x, const float* s) {
    launch(n, [&] { lsqr32::scal(n, pairs(x), pair(s)); });
}

}  // extern "C"
