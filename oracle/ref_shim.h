// OpenCL C built-ins for running the reference's own kernel text on the CPU — TEST INFRASTRUCTURE
// ONLY (the checker's strongest pin: the reference's code itself, not a restatement of it).
//
// The kernel strings of src/TomoStar.Core/Forward/EikonalOpenCl.cs:387-624 and
// src/TomoStar.Core/Numerics/LsqrOpenCl.cs:41-176 are extracted by oracle/ref_extract.py into
// oracle/_ref/ and compiled as C++ after this header, with -ffp-contract=off as their
// `#pragma OPENCL FP_CONTRACT OFF` demands. A launch is run as a loop over its work items in index
// order; the kernels driven here (eik_clear/seed/dirty/sweep, spmv and the vector updates) have
// work items that never read what another item of the same launch writes (eik_sweep's own comment:
// no node of a plane is another's neighbour), so any order gives the device's result.
//
// Arithmetic: the host's float and double operations are IEEE round-to-nearest (SSE2), and the
// float overloads of sqrt and fma are used for float arguments, as OpenCL's built-ins are typed.
// OpenCL lets a device's float divide and sqrt be up to 2.5 / 3 ulp off; the CPU rounds them
// correctly, which is what a conforming device with correctly rounded float division gives.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#define __kernel
#define __global
#define __local
#define __constant const
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

typedef unsigned char uchar;
typedef unsigned int uint;
typedef unsigned long ulong;
static_assert(sizeof(long) == 8, "OpenCL long is 64 bits");

using std::fma;
using std::isfinite;
using std::sqrt;

struct float2 {
    float x, y;
};
static inline float2 make_float2(float x, float y) {
    float2 r;
    r.x = x;
    r.y = y;
    return r;
}
static inline float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }

// Integer min/max of OpenCL C (the kernels use them on int only).
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }

// The NDRange position of the work item being run.
struct RefItem {
    size_t gid[2] = {0, 0};
    size_t lid[2] = {0, 0};
    size_t lsize[2] = {1, 1};
    size_t group[2] = {0, 0};
    size_t ngroups[2] = {1, 1};
};
extern thread_local RefItem ref_item;

static inline size_t get_global_id(int d) { return ref_item.gid[d]; }
static inline size_t get_local_id(int d) { return ref_item.lid[d]; }
static inline size_t get_local_size(int d) { return ref_item.lsize[d]; }
static inline size_t get_group_id(int d) { return ref_item.group[d]; }
static inline size_t get_num_groups(int d) { return ref_item.ngroups[d]; }

// A work-group barrier cannot be run by items executed one after another; the kernels that need it
// (dot_partial) are not driven on the CPU.
static inline void barrier(int) {
    std::fprintf(stderr, "ref_shim: barrier() reached; work-group kernels are not driven on the CPU\n");
    std::abort();
}

// Sequential items: the atomic is a plain read-modify-write.
static inline int atomic_or(volatile int* p, int v) {
    int old = *p;
    *p = old | v;
    return old;
}
