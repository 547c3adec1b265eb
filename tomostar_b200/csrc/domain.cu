// The forward domain and model (Forward/ForwardDomain.cs:24-107, Forward/TravelTimeTable.cs:213-241):
// the covering grid that holds stations and events outside the inversion grid, and the forward
// slowness resampled from the inversion grid on the device, with a fixed 1-D background outside it,
// straight into a resident model.
//
// Compiled with -fmad=false: the trilinear sums round term by term, as the reference's do.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "ctx.h"
#include "geo_dev.cuh"
#include "host_geo.h"

namespace ts {
namespace rays {
geo::RGrid make_rgrid(const host::Grid& g);
}

namespace domain {

using geo::RGrid;

// ForwardModel.FromInversionGrid (TravelTimeTable.cs:217-241) per forward node and phase: the
// velocity 1/s of the inversion grid interpolated at the node (SphericalGrid.Interpolate, all eight
// terms), the background's where the node lies outside the inversion grid (tolerance 1e-6), then 1/v.
template <typename Real>
__global__ void resample_kernel(const RGrid fg, const RGrid ig, const double* __restrict__ inv_s, int64_t inv_n,
                                int n_phases, int nbg, const double* __restrict__ bg_depth,
                                const double* __restrict__ bg_v, Real* __restrict__ out) {
    const int64_t fn = int64_t(fg.nx) * fg.ny * fg.nz;
    for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < fn;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const int i = int(idx % fg.nx), j = int((idx / fg.nx) % fg.ny), k = int(idx / (int64_t(fg.nx) * fg.ny));
        const double lon = fg.min_lon + i * fg.dlon, lat = fg.min_lat + j * fg.dlat, dep = fg.min_dep + k * fg.ddep;
        const bool outside = nbg > 0 && !geo::contains(ig, lon, lat, dep, 1e-6);
        double fx, fy, fz;
        geo::fractional(ig, lon, lat, dep, fx, fy, fz);
        int i0, j0, k0;
        double w[8];
        geo::weights(ig, fx, fy, fz, i0, j0, k0, w);
        const int64_t nxy = int64_t(ig.nx) * ig.ny;
        const int64_t base = k0 * nxy + int64_t(j0) * ig.nx + i0;
        for (int p = 0; p < n_phases; p++) {
            double v;
            if (outside) {
                v = geo::background_1d(bg_depth, bg_v + p * nbg, nbg, dep);
            } else {
                const double* s = inv_s + p * inv_n;
                double sum = 0;
                int n = 0;
#pragma unroll
                for (int dk = 0; dk < 2; dk++)
#pragma unroll
                    for (int dj = 0; dj < 2; dj++)
#pragma unroll
                        for (int di = 0; di < 2; di++) {
                            sum += (1 / s[base + dk * nxy + dj * ig.nx + di]) * w[n];
                            n++;
                        }
                v = sum;
            }
            out[p * fn + idx] = Real(1 / v);
        }
    }
}

}  // namespace domain
}  // namespace ts

using namespace ts;

extern "C" {

int ts_domain_covering(const ts_grid* inv, int32_t refinement, int32_t n_points, const double* points,
                       int64_t max_nodes, ts_grid* out, int32_t* extended, double* coarsening) {
    if (!inv || !out || (n_points > 0 && !points) || n_points < 0) {
        ts_thread_error() = "bad arguments";
        return TS_E_ARG;
    }
    if (const char* bad = host::Grid::validate(*inv)) {
        ts_thread_error() = bad;
        return TS_E_ARG;
    }
    if (inv->depth_km) {
        ts_thread_error() = "the covering domain needs a uniform inversion grid";
        return TS_E_ARG;
    }
    if (max_nodes <= 0) max_nodes = 12000000;
    // GridDefinition.Refined (Geo/SphericalGrid.cs:51-56).
    const int f = std::max(1, refinement);
    ts_grid fine = *inv;
    if (f > 1) {
        fine.nx = (inv->nx - 1) * f + 1;
        fine.ny = (inv->ny - 1) * f + 1;
        fine.nz = (inv->nz - 1) * f + 1;
    }
    const double fdlon = (fine.max_lon - fine.min_lon) / std::max(1, fine.nx - 1);
    const double fdlat = (fine.max_lat - fine.min_lat) / std::max(1, fine.ny - 1);
    const double fddep = (fine.max_depth_km - fine.min_depth_km) / std::max(1, fine.nz - 1);
    // ForwardDomain.Covering (Forward/ForwardDomain.cs:51-107).
    const double centre = 0.5 * (inv->min_lon + inv->max_lon);
    double min_lon = inv->min_lon, max_lon = inv->max_lon, min_lat = inv->min_lat, max_lat = inv->max_lat;
    const double top = inv->min_depth_km;
    double bottom = inv->max_depth_km;
    int outside = 0;
    for (int q = 0; q < n_points; q++) {
        const double lon = host::unwrap_lon(points[3 * q], centre), lat = points[3 * q + 1], dep = points[3 * q + 2];
        const bool inside = lon >= inv->min_lon && lon <= inv->max_lon && lat >= inv->min_lat && lat <= inv->max_lat &&
                            dep >= inv->min_depth_km && dep <= inv->max_depth_km;
        if (inside) continue;
        outside++;
        min_lon = std::min(min_lon, lon);
        max_lon = std::max(max_lon, lon);
        min_lat = std::min(min_lat, lat);
        max_lat = std::max(max_lat, lat);
        bottom = std::max(bottom, dep);  // stations above the top are placed on it
    }
    if (extended) *extended = outside > 0;
    if (coarsening) *coarsening = 1.0;
    if (outside == 0) {
        *out = fine;
        out->depth_km = nullptr;
        return TS_OK;
    }
    min_lon -= 2 * fdlon;
    max_lon += 2 * fdlon;
    min_lat = std::max(-89.0, min_lat - 2 * fdlat);
    max_lat = std::min(89.0, max_lat + 2 * fdlat);
    if (bottom > inv->max_depth_km) bottom += 2 * fddep;
    if (max_lon - min_lon >= 359) {
        ts_thread_error() = "Stations and events outside the area span the whole globe: restrict the data.";
        return TS_E_ARG;
    }
    double dlon = fdlon, dlat = fdlat, ddep = fddep;
    auto count = [&](double fc) {
        return int64_t(std::ceil((max_lon - min_lon) / (dlon * fc)) + 1) *
               int64_t(std::ceil((max_lat - min_lat) / (dlat * fc)) + 1) *
               int64_t(std::ceil((bottom - top) / (ddep * fc)) + 1);
    };
    double factor = 1.0;
    while (count(factor) > max_nodes) factor *= 1.25;
    dlon *= factor;
    dlat *= factor;
    ddep *= factor;
    const int west = int(std::ceil((inv->min_lon - min_lon) / dlon)), east = int(std::ceil((max_lon - inv->max_lon) / dlon));
    const int south = int(std::ceil((inv->min_lat - min_lat) / dlat)), north = int(std::ceil((max_lat - inv->max_lat) / dlat));
    const int down = int(std::ceil((bottom - inv->max_depth_km) / ddep));
    // Math.Round is to even, as nearbyint.
    const int nx = int(std::nearbyint((inv->max_lon - inv->min_lon) / dlon));
    const int ny = int(std::nearbyint((inv->max_lat - inv->min_lat) / dlat));
    const int nz = int(std::nearbyint((inv->max_depth_km - inv->min_depth_km) / ddep));
    ts_grid d{};
    d.min_lon = inv->min_lon - west * dlon;
    d.max_lon = inv->min_lon - west * dlon + (west + nx + east) * dlon;
    d.min_lat = inv->min_lat - south * dlat;
    d.max_lat = inv->min_lat - south * dlat + (south + ny + north) * dlat;
    d.min_depth_km = inv->min_depth_km;
    d.max_depth_km = inv->min_depth_km + (nz + down) * ddep;
    d.nx = west + nx + east + 1;
    d.ny = south + ny + north + 1;
    d.nz = nz + down + 1;
    d.depth_km = nullptr;
    if (const char* bad = host::Grid::validate(d)) {
        ts_thread_error() = bad;
        return TS_E_ARG;
    }
    *out = d;
    if (coarsening) *coarsening = factor;
    return TS_OK;
}

int ts_model_put_resampled(ts_ctx* ctx, const ts_grid* forward, const ts_grid* inversion, const double* inv_slowness,
                           int32_t n_phases, const ts_background* bg, int32_t precision, int32_t* model_id) {
    if (!ctx || !model_id) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    *model_id = 0;
    if (!forward || !inversion || !inv_slowness || n_phases <= 0 || n_phases > 2)
        return ctx->fail(TS_E_ARG, "bad arguments (one or two phases)");
    if (const char* bad = host::Grid::validate(*forward)) return ctx->fail(TS_E_ARG, bad);
    if (const char* bad = host::Grid::validate(*inversion)) return ctx->fail(TS_E_ARG, bad);
    if (forward->depth_km || inversion->depth_km) return ctx->fail(TS_E_ARG, "resampling needs uniform grids");
    if (precision != TS_PRECISION_F64 && precision != TS_PRECISION_F32) return ctx->fail(TS_E_ARG, "precision");
    const int nbg = bg ? bg->n : 0;
    if (nbg < 0 || (nbg > 0 && (!bg->depth_km || !bg->vp || !bg->vs)))
        return ctx->fail(TS_E_ARG, "bad background model");
    auto* m = new ts_ctx::Model();
    m->def = *forward;
    m->grid = new host::Grid(m->def);
    m->metric = new host::Metric(*m->grid);
    m->precision = precision;
    m->n_phases = n_phases;
    const host::Grid ig(*inversion);
    const int64_t fn = m->grid->count(), in = ig.count();
    const size_t esz = 8;  // a double, or the float pair of the FP32 precision
    if (cudaMalloc(&m->slowness, size_t(fn) * n_phases * esz) != cudaSuccess) {
        cudaGetLastError();
        m->slowness = nullptr;
        delete m;
        return ctx->fail(TS_E_NOMEM, "model slowness");
    }
    double* s_d = static_cast<double*>(ctx->buf("dom.inv_slowness", sizeof(double) * size_t(in) * n_phases));
    double* bg_d = static_cast<double*>(ctx->buf("dom.background", sizeof(double) * 3 * std::max(1, nbg)));
    if (!s_d || !bg_d) {
        delete m;
        return TS_E_NOMEM;
    }
    std::vector<double> bgv(3 * std::max(1, nbg));
    for (int q = 0; q < nbg; q++) {
        bgv[q] = bg->depth_km[q];
        bgv[nbg + q] = bg->vp[q];
        bgv[2 * nbg + q] = bg->vs[q];
    }
    cudaStream_t s = ctx->stream;
    int rc = TS_OK;
    if (cudaMemcpyAsync(s_d, inv_slowness, sizeof(double) * size_t(in) * n_phases, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(bg_d, bgv.data(), sizeof(double) * bgv.size(), cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = TS_E_CUDA;
    const geo::RGrid fg = rays::make_rgrid(*m->grid), rg = rays::make_rgrid(ig);
    const int blocks = int(std::min<int64_t>((fn + 255) / 256, int64_t(ctx->sm_count) * 16));
    if (!rc) {
        if (precision == TS_PRECISION_F64)
            domain::resample_kernel<double><<<blocks, 256, 0, s>>>(fg, rg, s_d, in, n_phases, nbg, bg_d, bg_d + nbg,
                                                                   static_cast<double*>(m->slowness));
        else
            domain::resample_kernel<Pair><<<blocks, 256, 0, s>>>(fg, rg, s_d, in, n_phases, nbg, bg_d, bg_d + nbg,
                                                                 static_cast<Pair*>(m->slowness));
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) rc = TS_E_CUDA;
    }
    if (rc) {
        delete m;
        return ctx->fail(rc, "resampling failed");
    }
    *model_id = ctx->next_model++;
    ctx->models[*model_id] = m;
    return TS_OK;
}

int ts_model_copy_slowness(ts_ctx* ctx, int32_t model_id, int32_t phase, double* out) {
    if (!ctx || !out) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    auto it = ctx->models.find(model_id);
    if (it == ctx->models.end()) return ctx->fail(TS_E_ARG, "unknown model");
    ts_ctx::Model* m = it->second;
    if (phase < 0 || phase >= m->n_phases) return ctx->fail(TS_E_ARG, "phase out of range");
    const size_t n = size_t(m->grid->count());
    if (m->precision == TS_PRECISION_F64) {
        TS_CUDA_TRY(ctx, cudaMemcpy(out, static_cast<double*>(m->slowness) + n * phase, n * 8, cudaMemcpyDeviceToHost));
    } else {
        // The FP32 precision's slowness is the float the paired kernel reads (the pair's hi).
        std::vector<Pair> tmp(n);
        TS_CUDA_TRY(ctx, cudaMemcpy(tmp.data(), static_cast<Pair*>(m->slowness) + n * phase, n * sizeof(Pair),
                                    cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < n; q++) out[q] = tmp[q].hi;
    }
    return TS_OK;
}

int ts_set_background(ts_ctx* ctx, const ts_background* bg) {
    if (!ctx) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!bg || bg->n == 0) {
        ctx->bg_n = 0;
        return TS_OK;
    }
    if (bg->n < 0 || !bg->depth_km || !bg->vp || !bg->vs) return ctx->fail(TS_E_ARG, "bad background model");
    for (int q = 0; q < bg->n; q++)
        if (!(bg->vp[q] > 0) || !(bg->vs[q] > 0) || (q > 0 && bg->depth_km[q] < bg->depth_km[q - 1]))
            return ctx->fail(TS_E_ARG, "background velocities must be positive and depths non-decreasing");
    std::vector<double> v(3 * size_t(bg->n));
    for (int q = 0; q < bg->n; q++) {
        v[q] = bg->depth_km[q];
        v[bg->n + q] = bg->vp[q];
        v[2 * bg->n + q] = bg->vs[q];
    }
    double* d = static_cast<double*>(ctx->buf("rays.background", sizeof(double) * v.size()));
    if (!d) return TS_E_NOMEM;
    TS_CUDA_TRY(ctx, cudaMemcpy(d, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice));
    ctx->bg_n = bg->n;
    return TS_OK;
}

}  // extern "C"
