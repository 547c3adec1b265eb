// The reference's device eikonal (EikonalOpenCl.cs) run on the CPU from its own kernel text —
// TEST INFRASTRUCTURE ONLY.
//
// Compiled twice by oracle/Makefile: with -DQV_FP64 (the double kernel, exported as ref_eik_solve_f64)
// and without (times as float pairs hi + lo, exported as ref_eik_solve_paired). The kernel source is
// the `Kernel` literal of src/TomoStar.Core/Forward/EikonalOpenCl.cs:387-624, extracted into
// oracle/_ref/eik_kernel.cl by oracle/ref_extract.py; this file adds only the host side:
//
// * TrySolve's seed handling (EikonalOpenCl.cs:138-166): out-of-range seeds dropped, duplicates keep
//   the smallest time, positions node-major (node · batch + field);
// * Sweep's launch sequence (EikonalOpenCl.cs:167-300): eik_clear, eik_seed, then per phase
//   (eik_dirty before phase 1) rounds of 8 orderings × planes of one eik_sweep launch each, the
//   changed flag zeroed before and read after every round, refusal when a phase has not settled
//   within SphericalEikonal.SweepRoundCap; the uploads in the device's precision (UploadReal,
//   UploadTime) and the read-back (double, or hi + lo summed as double);
// * the NDRange of each launch as Sweep sets it (LocalSize 64, global sizes rounded up), run as a
//   loop over the work items.
#include <algorithm>
#include <map>
#include <vector>

#include "ref_shim.h"

#ifdef QV_FP64
#define REF_NS ref64
#define REF_SOLVE ref_eik_solve_f64
#else
#define REF_NS ref32
#define REF_SOLVE ref_eik_solve_paired
#endif

namespace REF_NS {
#include "eik_kernel.cl"
}

namespace {

constexpr size_t kLocalSize = 64;  // EikonalOpenCl.LocalSize

size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

// SphericalEikonal.PlaneBounds (SphericalEikonal.cs:339-346).
void plane_bounds(int nx, int ny, int nz, int p, int& i0, int& i1, int& k0, int& k1) {
    i0 = std::max(0, p - (ny - 1) - (nz - 1));
    i1 = std::min(nx - 1, p);
    k0 = std::max(0, p - (nx - 1) - (ny - 1));
    k1 = std::min(nz - 1, p);
}

template <typename F>
void run_1d(size_t global, F&& body) {
    for (size_t q = 0; q < global; q++) {
        ref_item.gid[0] = q;
        ref_item.gid[1] = 0;
        body();
    }
}

using REF_NS::real;
using REF_NS::tval;

// UploadTime: a time in the device's precision (a double, or hi + lo).
tval to_tval(double t) {
#ifdef QV_FP64
    return t;
#else
    float hi = (float)t;
    float lo = std::isfinite(hi) ? (float)(t - (double)hi) : 0.0f;
    return make_float2(hi, lo);
#endif
}

double from_tval(tval v) {
#ifdef QV_FP64
    return v;
#else
    return (double)v.x + (double)v.y;
#endif
}

}  // namespace

extern "C" {

// Solves `batch` fields on one grid. hlon[ny·nz], hlat[nz], hr: GridMetric (SphericalEikonal.cs:15-35).
// Seeds of field e are seed_idx/seed_time[seed_off[e] .. seed_off[e+1]). out: batch·n doubles,
// field-major. rounds[2]: rounds per phase. cap <= 0 takes SweepRoundCap. Returns 0 when settled,
// 1 when a phase did not settle within the cap, 2 when no seed is on the grid.
int REF_SOLVE(int nx, int ny, int nz, const double* hlon, const double* hlat, double hr, const double* slowness,
              int batch, const int32_t* seed_off, const int32_t* seed_idx, const double* seed_time, int cap,
              double* out, int32_t* rounds) {
    const long n = (long)nx * ny * nz;
    const long total = (long)batch * n;
    // TrySolve: merge per field, node-major positions.
    std::vector<long> at;
    std::vector<tval> tt;
    for (int e = 0; e < batch; e++) {
        std::map<int, double> merged;
        for (int q = seed_off[e]; q < seed_off[e + 1]; q++) {
            if ((unsigned)seed_idx[q] >= (unsigned)n) continue;
            auto it = merged.find(seed_idx[q]);
            if (it == merged.end() || seed_time[q] < it->second) merged[seed_idx[q]] = seed_time[q];
        }
        for (auto& kv : merged) {
            at.push_back((long)kv.first * batch + e);
            tt.push_back(to_tval(kv.second));
        }
    }
    if (at.empty()) return 2;
    // UploadReal: slowness and metric in the device's precision.
    std::vector<real> s(n), hl((size_t)ny * nz), ht(nz);
    for (long q = 0; q < n; q++) s[q] = (real)slowness[q];
    for (size_t q = 0; q < hl.size(); q++) hl[q] = (real)hlon[q];
    for (int q = 0; q < nz; q++) ht[q] = (real)hlat[q];
    const real hrr = (real)hr;
    std::vector<tval> f(total);
    std::vector<uchar> seeded(total), dirty(total);
    int changed = 0;

    const size_t clear_global = round_up(total, kLocalSize);
    run_1d(clear_global, [&] { REF_NS::eik_clear(f.data(), seeded.data(), dirty.data(), total); });
    const int count = (int)at.size();
    run_1d((size_t)count, [&] { REF_NS::eik_seed(f.data(), seeded.data(), at.data(), tt.data(), count); });

    if (cap <= 0) cap = std::max(32, (nx + ny + nz) / 4);  // SphericalEikonal.SweepRoundCap
    const int planes = nx + ny + nz - 2;
    int status = 0;
    for (int phase = 0; phase < 2 && status == 0; phase++) {
        if (phase > 0) run_1d(clear_global, [&] { REF_NS::eik_dirty(dirty.data(), total); });
        bool settled = false;
        for (int round = 0; round < cap && !settled; round++) {
            changed = 0;
            for (int dir = 0; dir < 8; dir++)
                for (int p = 0; p < planes; p++) {
                    int i0, i1, k0, k1;
                    plane_bounds(nx, ny, nz, p, i0, i1, k0, k1);
                    const long items = (long)(i1 - i0 + 1) * batch;
                    const size_t g0 = round_up((size_t)items, kLocalSize), g1 = (size_t)(k1 - k0 + 1);
                    for (size_t y = 0; y < g1; y++)
                        for (size_t x = 0; x < g0; x++) {
                            ref_item.gid[0] = x;
                            ref_item.gid[1] = y;
                            REF_NS::eik_sweep(f.data(), s.data(), hl.data(), ht.data(), hrr, seeded.data(), nx, ny, nz,
                                              phase, &changed, dir, p, batch, dirty.data());
                        }
                }
            rounds[phase] = round + 1;
            settled = changed == 0;
        }
        if (!settled) status = 1;
    }
    // Back to field-major.
    for (int e = 0; e < batch; e++)
        for (long q = 0; q < n; q++) out[(long)e * n + q] = from_tval(f[q * batch + e]);
    return status;
}

}  // extern "C"
