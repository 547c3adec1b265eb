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

template <typename Real>
TS_HDINL Real real_inf();
template <>
TS_HDINL double real_inf<double>() { return __builtin_huge_val(); }
template <>
TS_HDINL float real_inf<float>() { return __builtin_huge_valf(); }

// Loads that bypass L1: values other SMs rewrite between two barriers of one launch.
TS_DEVINL float ld_cg(const float* p) { return __ldcg(p); }
TS_DEVINL double ld_cg(const double* p) { return __ldcg(p); }
TS_DEVINL void st_cg(float* p, float v) { __stcg(p, v); }
TS_DEVINL void st_cg(double* p, double v) { __stcg(p, v); }

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
TS_DEVINL void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

}  // namespace ts
