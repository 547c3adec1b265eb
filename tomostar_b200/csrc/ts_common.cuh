// Shared definitions of the CUDA forward engine: constants, error codes, small device helpers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/tomostar_cuda.h"

#define TS_DEVINL __device__ __forceinline__
#define TS_HDINL __host__ __device__ __forceinline__

namespace ts {

constexpr double kEarthRadiusKm = 6371.0;  // Geo/GeoMath.cs:43
constexpr double kDeg2Rad = 3.14159265358979323846 / 180.0;
constexpr double kRad2Deg = 180.0 / 3.14159265358979323846;

// SphericalEikonal.SettleTolerance (Forward/SphericalEikonal.cs:332).
constexpr double kSettleTolerance = 1e-7;

TS_HDINL double dinf() { return __builtin_huge_val(); }

// The FP32 precision's value type: a time as two floats hi + lo (about 48 bits in the 8 bytes of a
// double), the reference's field type on devices without FP64 (EikonalOpenCl.cs:29-37, 409-413).
// Slowness and axis weights are carried in the same type with only hi used (lo = 0 for weights;
// the reference narrows them to float, EikonalOpenCl.cs:320-333).
//
// Conversions follow the reference's host: from a double, hi = (float)v and lo = (float)(v − hi)
// when hi is finite, else 0 (UploadTime, EikonalOpenCl.cs:303-317); back to a double, hi + lo in
// double (the read-back, EikonalOpenCl.cs:289-293).
//
// Order: `a < b` is the reference's acceptance test written as a comparison, the paired difference
// (b.hi − a.hi) + (b.lo − a.lo) rounded in float being > 0 (eik_sweep's `drop > 0`); with +inf in b
// (lo 0) that is true for every finite a. It is used where the engine decides that a candidate
// replaces a held time and where a causal wake compares a neighbour with a new time.
struct __align__(8) Pair {
    float hi, lo;
    Pair() = default;
    TS_HDINL Pair(float h, float l) : hi(h), lo(l) {}
    TS_HDINL explicit Pair(double v) {
        hi = float(v);
        lo = (hi - hi == 0.0f) ? float(v - double(hi)) : 0.0f;  // hi − hi is 0 exactly when hi is finite
    }
    TS_HDINL explicit Pair(int v) : hi(float(v)), lo(0.0f) {}
    TS_HDINL explicit operator double() const { return double(hi) + double(lo); }
    TS_HDINL explicit operator float() const { return float(double(hi) + double(lo)); }
};

// The paired difference a − b as one float (the reference's df_sub, EikonalOpenCl.cs:460): exact in
// the hi part for neighbouring times (Sterbenz), +inf when a is +inf and b finite.
TS_HDINL float pair_sub(Pair a, Pair b) { return (a.hi - b.hi) + (a.lo - b.lo); }
TS_HDINL bool operator<(Pair a, Pair b) { return pair_sub(b, a) > 0.0f; }

// Finite test of a value of any of the value types (a Pair by its hi part, as the reference does).
TS_HDINL bool finite_r(double v) { return v - v == 0.0; }
TS_HDINL bool finite_r(float v) { return v - v == 0.0f; }
TS_HDINL bool finite_r(Pair v) { return v.hi - v.hi == 0.0f; }

template <typename Real>
TS_HDINL Real real_inf();
template <>
TS_HDINL double real_inf<double>() { return __builtin_huge_val(); }
template <>
TS_HDINL float real_inf<float>() { return __builtin_huge_valf(); }
template <>
TS_HDINL Pair real_inf<Pair>() { return Pair(__builtin_huge_valf(), 0.0f); }

// The C ABI precision a field value type stands for: FP64 fields are double, FP32 fields are Pair.
template <typename Real>
struct PrecisionOf;
template <>
struct PrecisionOf<double> {
    static constexpr int value = TS_PRECISION_F64;
};
template <>
struct PrecisionOf<Pair> {
    static constexpr int value = TS_PRECISION_F32;
};
template <typename Real>
TS_HDINL constexpr int precision_of() { return PrecisionOf<Real>::value; }
template <typename Real>
TS_HDINL constexpr bool is_f64() { return PrecisionOf<Real>::value == TS_PRECISION_F64; }

// An axis weight in a precision's own arithmetic: the FP64 kernel's double weight, or the paired
// kernel's float weight (computed in float from the narrowed spacing, EikonalOpenCl.cs:492-495),
// carried as a double that converts to the value type exactly.
template <typename Real>
TS_HDINL double weight_of(double w64, float w32) { return is_f64<Real>() ? w64 : double(w32); }

// Loads that bypass L1: values other SMs rewrite between two barriers of one launch.
TS_DEVINL float ld_cg(const float* p) { return __ldcg(p); }
TS_DEVINL double ld_cg(const double* p) { return __ldcg(p); }
TS_DEVINL Pair ld_cg(const Pair* p) {
    float2 v = __ldcg(reinterpret_cast<const float2*>(p));
    return Pair(v.x, v.y);
}
TS_DEVINL void st_cg(float* p, float v) { __stcg(p, v); }
TS_DEVINL void st_cg(double* p, double v) { __stcg(p, v); }
TS_DEVINL void st_cg(Pair* p, Pair v) { __stcg(reinterpret_cast<float2*>(p), make_float2(v.hi, v.lo)); }

// Read-only loads through the non-coherent path.
TS_DEVINL float ldg_r(const float* p) { return __ldg(p); }
TS_DEVINL double ldg_r(const double* p) { return __ldg(p); }
TS_DEVINL Pair ldg_r(const Pair* p) {
    float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return Pair(v.x, v.y);
}

// Warp shuffles of a value (a Pair moves as its two floats).
TS_DEVINL double shfl_up_r(unsigned m, double v, int d) { return __shfl_up_sync(m, v, d); }
TS_DEVINL double shfl_down_r(unsigned m, double v, int d) { return __shfl_down_sync(m, v, d); }
TS_DEVINL float shfl_up_r(unsigned m, float v, int d) { return __shfl_up_sync(m, v, d); }
TS_DEVINL float shfl_down_r(unsigned m, float v, int d) { return __shfl_down_sync(m, v, d); }
TS_DEVINL Pair shfl_up_r(unsigned m, Pair v, int d) {
    return Pair(__shfl_up_sync(m, v.hi, d), __shfl_up_sync(m, v.lo, d));
}
TS_DEVINL Pair shfl_down_r(unsigned m, Pair v, int d) {
    return Pair(__shfl_down_sync(m, v.hi, d), __shfl_down_sync(m, v.lo, d));
}

// Asynchronous global → shared copies (LDGSTS): a warp issues every copy of a tile before it
// waits once, instead of one round trip per loop iteration. The 16-byte .cg form bypasses L1, so it
// never serves a line another SM has rewritten since; the 4/8-byte .ca form is for read-only data.
TS_DEVINL void cp_async16_cg(void* smem, const void* gmem) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
TS_DEVINL void cp_async_ro(float* smem, const float* gmem) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
TS_DEVINL void cp_async_ro(double* smem, const double* gmem) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
TS_DEVINL void cp_async_ro(Pair* smem, const Pair* gmem) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
TS_DEVINL void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

}  // namespace ts
