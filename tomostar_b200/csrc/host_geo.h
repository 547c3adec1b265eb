// Host-side geometry of the C ABI: the spherical grid, its eikonal metric and the point-source
// seeds, as the reference computes them on the host before a device solve. Compiled with
// -ffp-contract=off so the doubles are the reference's (glibc libm, as .NET on Linux).
//
// Also the host sweeping solver the self-test gate compares the device against
// (EikonalOpenCl.SelfTest runs SphericalEikonal.Relax on the host, EikonalOpenCl.cs:359). It is
// used by ts_cuda_selftest only and never produces a solve's result.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

#include "../../include/tomostar_cuda.h"

namespace ts {
namespace host {

constexpr double kEarthRadiusKm = 6371.0;  // Geo/GeoMath.cs:43
constexpr double kDeg2Rad = M_PI / 180.0;  // Geo/GeoMath.cs:45
constexpr double kInf = std::numeric_limits<double>::infinity();

struct V3 {
    double x, y, z;
};

// GeoMath.ToCartesian (Geo/GeoMath.cs:49-56).
inline V3 to_cartesian(double lon_deg, double lat_deg, double depth_km) {
    double r = kEarthRadiusKm - depth_km;
    double lat = lat_deg * kDeg2Rad, lon = lon_deg * kDeg2Rad;
    double cl = std::cos(lat);
    return {r * cl * std::cos(lon), r * cl * std::sin(lon), r * std::sin(lat)};
}
inline double dist(V3 a, V3 b) {
    double x = a.x - b.x, y = a.y - b.y, z = a.z - b.z;
    return std::sqrt(x * x + y * y + z * z);
}

// GeoMath.UnwrapLon (Geo/GeoMath.cs:146-151).
inline double unwrap_lon(double lon, double ref) {
    if (lon < ref - 180) lon += 360 * std::ceil((ref - 180 - lon) / 360);
    else if (lon > ref + 180) lon -= 360 * std::ceil((lon - ref - 180) / 360);
    return lon;
}

// SphericalGrid (Geo/SphericalGrid.cs:84-116) with the variable-depth extension.
struct Grid {
    int nx = 0, ny = 0, nz = 0;
    double min_lon = 0, min_lat = 0, min_dep = 0, dlon = 0, dlat = 0, ddep = 0;
    double centre_lon = 0, dlon_rad = 0, dlat_rad = 0;
    bool variable = false;
    std::vector<double> lon, lat, coslat, dep, rad;

    // GridDefinition.Validate (SphericalGrid.cs:33-44); returns an error text or null.
    static const char* validate(const ts_grid& d) {
        if (!std::isfinite(d.min_lon) || !std::isfinite(d.max_lon) || !std::isfinite(d.min_lat) ||
            !std::isfinite(d.max_lat) || !std::isfinite(d.min_depth_km) || !std::isfinite(d.max_depth_km))
            return "Grid bounds must be finite.";
        if (d.nx < 2 || d.ny < 2 || d.nz < 2) return "A grid needs at least two nodes on every axis.";
        if (!(d.max_lon > d.min_lon) || !(d.max_lat > d.min_lat) || !(d.max_depth_km > d.min_depth_km))
            return "Grid bounds are empty or inverted.";
        if (d.max_lon - d.min_lon >= 360) return "A grid must span less than 360 degrees of longitude.";
        if (d.min_lat < -89.9 || d.max_lat > 89.9) return "Grids touching the poles are not supported.";
        if (d.max_depth_km >= kEarthRadiusKm) return "The grid reaches the centre of the Earth.";
        if (int64_t(d.nx) * d.ny * d.nz > int64_t(INT32_MAX)) return "Grid has more than 2^31 nodes.";
        if (d.depth_km) {
            for (int k = 0; k + 1 < d.nz; k++)
                if (!(d.depth_km[k + 1] > d.depth_km[k])) return "Grid depths must increase.";
        }
        return nullptr;
    }

    explicit Grid(const ts_grid& d) {
        nx = d.nx; ny = d.ny; nz = d.nz;
        min_lon = d.min_lon; min_lat = d.min_lat; min_dep = d.min_depth_km;
        dlon = (d.max_lon - d.min_lon) / std::max(1, nx - 1);
        dlat = (d.max_lat - d.min_lat) / std::max(1, ny - 1);
        ddep = (d.max_depth_km - d.min_depth_km) / std::max(1, nz - 1);
        variable = d.depth_km != nullptr;
        lon.resize(nx); lat.resize(ny); coslat.resize(ny); dep.resize(nz); rad.resize(nz);
        for (int i = 0; i < nx; i++) lon[i] = d.min_lon + i * dlon;
        for (int j = 0; j < ny; j++) {
            lat[j] = d.min_lat + j * dlat;
            coslat[j] = std::cos(lat[j] * kDeg2Rad);
        }
        for (int k = 0; k < nz; k++) {
            dep[k] = variable ? d.depth_km[k] : d.min_depth_km + k * ddep;
            rad[k] = kEarthRadiusKm - dep[k];
        }
        centre_lon = 0.5 * (d.min_lon + d.max_lon);
        dlon_rad = dlon * kDeg2Rad;
        dlat_rad = dlat * kDeg2Rad;
    }
    int64_t count() const { return int64_t(nx) * ny * nz; }
    int index(int i, int j, int k) const { return (k * ny + j) * nx + i; }

    double frac_z(double depth_km) const {
        if (!variable) return (depth_km - min_dep) / ddep;
        if (depth_km <= dep[0]) return (depth_km - dep[0]) / (dep[1] - dep[0]);
        if (depth_km >= dep[nz - 1]) return (nz - 1) + (depth_km - dep[nz - 1]) / (dep[nz - 1] - dep[nz - 2]);
        int k = int(std::upper_bound(dep.begin(), dep.end(), depth_km) - dep.begin()) - 1;
        return k + (depth_km - dep[k]) / (dep[k + 1] - dep[k]);
    }
    // SphericalGrid.Fractional (SphericalGrid.cs:179-184).
    void fractional(double lo, double la, double de, double& fx, double& fy, double& fz) const {
        if (lo < centre_lon - 180 || lo > centre_lon + 180) lo = unwrap_lon(lo, centre_lon);
        fx = (lo - min_lon) / dlon;
        fy = (la - min_lat) / dlat;
        fz = frac_z(de);
    }
    // SphericalGrid.Interpolate via TrilinearWeightsFractional (SphericalGrid.cs:205-235).
    double interpolate(const double* f, double lo, double la, double de) const {
        double fx, fy, fz;
        fractional(lo, la, de, fx, fy, fz);
        fx = std::clamp(fx, 0.0, double(nx - 1));
        fy = std::clamp(fy, 0.0, double(ny - 1));
        fz = std::clamp(fz, 0.0, double(nz - 1));
        int i0 = std::min(int(fx), nx - 2), j0 = std::min(int(fy), ny - 2), k0 = std::min(int(fz), nz - 2);
        double tx = fx - i0, ty = fy - j0, tz = fz - k0;
        double sum = 0;
        for (int dk = 0; dk < 2; dk++)
            for (int dj = 0; dj < 2; dj++)
                for (int di = 0; di < 2; di++) {
                    double w = (di == 0 ? 1 - tx : tx) * (dj == 0 ? 1 - ty : ty) * (dk == 0 ? 1 - tz : tz);
                    sum += f[index(i0 + di, j0 + dj, k0 + dk)] * w;
                }
        return sum;
    }
    // SphericalGrid.MinSpacingKm (SphericalGrid.cs:159-164).
    double min_spacing_km() const {
        double r_min = rad[nz - 1];
        double cos_min = *std::min_element(coslat.begin(), coslat.end());
        double dz = ddep;
        if (variable) {
            dz = kInf;
            for (int k = 0; k + 1 < nz; k++) dz = std::min(dz, dep[k + 1] - dep[k]);
        }
        return std::min(dz, std::min(r_min * dlat_rad, r_min * cos_min * dlon_rad));
    }
};

// GridMetric (Forward/SphericalEikonal.cs:15-35), the axis weights of the upwind terms and the
// per-level z coefficients of the extension (layout documented in eik_update.cuh). The weights are
// the reference's own divisions (SphericalEikonal.cs:369, 391): w1 = 1.0 / (h * h) first order,
// w2 = 1.0 / (he * he) with he = 2 * h / 3 second order, computed once per axis and level.
struct Metric {
    std::vector<double> hlon, hlat, zc;
    std::vector<double> wx;  // 2 per (k, j): w1, w2 of the longitude axis
    std::vector<double> wy;  // 2 per k: latitude axis
    double hr = 0, wz1 = 1, wz2 = 1;
    // The same weights as the paired-float kernel forms them, in float from the spacing narrowed to
    // float (eik_term: he = 2.0f * h / 3.0f, we = 1.0f / (he * he); EikonalOpenCl.cs:490-495).
    std::vector<float> wx32, wy32;
    float wz1_32 = 1, wz2_32 = 1;
    static void weights(double h, double& w1, double& w2) {
        w1 = 1.0 / (h * h);
        double he = 2 * h / 3;
        w2 = 1.0 / (he * he);
    }
    static void weights32(double h64, float& w1, float& w2) {
        const float h = float(h64);
        w1 = 1.0f / (h * h);
        const float he = 2.0f * h / 3.0f;
        w2 = 1.0f / (he * he);
    }
    explicit Metric(const Grid& g) {
        hlon.resize(size_t(g.ny) * g.nz);
        hlat.resize(g.nz);
        wx.resize(2 * hlon.size());
        wy.resize(2 * size_t(g.nz));
        wx32.resize(wx.size());
        wy32.resize(wy.size());
        for (int k = 0; k < g.nz; k++) {
            hlat[k] = g.rad[k] * g.dlat_rad;
            weights(hlat[k], wy[2 * k], wy[2 * k + 1]);
            weights32(hlat[k], wy32[2 * k], wy32[2 * k + 1]);
            for (int j = 0; j < g.ny; j++) {
                size_t q = size_t(k) * g.ny + j;
                hlon[q] = std::max(1e-9, g.rad[k] * g.coslat[j] * g.dlon_rad);
                weights(hlon[q], wx[2 * q], wx[2 * q + 1]);
                weights32(hlon[q], wx32[2 * q], wx32[2 * q + 1]);
            }
        }
        hr = g.ddep;
        weights(hr, wz1, wz2);
        weights32(hr, wz1_32, wz2_32);
        if (g.variable) {
            zc.assign(size_t(16) * g.nz, 1.0);
            auto side = [&](double* c, double h1, double h2) {
                double a = (2 * h1 + h2) / (h1 * (h1 + h2));
                double b = (h1 + h2) / (h1 * h2);
                double cc = h1 / (h2 * (h1 + h2));
                double he = 1 / a;
                c[0] = 1.0 / (h1 * h1); c[1] = 1.0 / (he * he); c[2] = a; c[3] = b; c[4] = cc; c[5] = cc / a;
            };
            for (int k = 0; k < g.nz; k++) {
                double* c = &zc[size_t(16) * k];
                double hm = k > 0 ? g.dep[k] - g.dep[k - 1] : 1.0;
                double hm2 = k > 1 ? g.dep[k - 1] - g.dep[k - 2] : hm;
                double hp = k + 1 < g.nz ? g.dep[k + 1] - g.dep[k] : 1.0;
                double hp2 = k + 2 < g.nz ? g.dep[k + 2] - g.dep[k + 1] : hp;
                side(c, hm, hm2);
                side(c + 8, hp, hp2);
            }
        }
    }
};

// SphericalEikonal.PointSource (Forward/SphericalEikonal.cs:68-100); the variable-depth
// extension takes the vertical spacing at the source and widens the depth search by two levels.
inline int point_source(const Grid& g, const double* slowness, double lon, double lat, double depth_km,
                        double origin_time, double radius_cells, int32_t* idx_out, double* t_out, int cap) {
    double dep = std::clamp(depth_km, g.dep[0], g.dep[g.nz - 1]);
    double fx, fy, fz;
    g.fractional(lon, lat, dep, fx, fy, fz);
    fx = std::clamp(fx, 0.0, double(g.nx - 1));
    fy = std::clamp(fy, 0.0, double(g.ny - 1));
    fz = std::clamp(fz, 0.0, double(g.nz - 1));
    V3 src = to_cartesian(lon, lat, dep);
    double s_src = g.interpolate(slowness, lon, lat, dep);
    double r = kEarthRadiusKm - dep;
    double h_lon = std::max(1e-9, r * std::cos(lat * kDeg2Rad) * g.dlon_rad);
    double h_lat = r * g.dlat_rad;
    double h_r = g.ddep;
    if (g.variable) {
        int kk = std::min(int(fz), g.nz - 2);
        h_r = g.dep[kk + 1] - g.dep[kk];
    }
    double radius_km = radius_cells * std::max(h_lon, std::max(h_lat, h_r));
    int ri = int(std::ceil(radius_km / h_lon)), rj = int(std::ceil(radius_km / h_lat)), rk = int(std::ceil(radius_km / h_r));
    if (g.variable) rk += 2;
    int i0 = int(std::nearbyint(fx)), j0 = int(std::nearbyint(fy)), k0 = int(std::nearbyint(fz));  // Math.Round: to even
    int n = 0;
    for (int k = std::max(0, k0 - rk); k <= std::min(g.nz - 1, k0 + rk); k++)
        for (int j = std::max(0, j0 - rj); j <= std::min(g.ny - 1, j0 + rj); j++)
            for (int i = std::max(0, i0 - ri); i <= std::min(g.nx - 1, i0 + ri); i++) {
                int idx = g.index(i, j, k);
                double d = dist(to_cartesian(g.lon[i], g.lat[j], g.dep[k]), src);
                bool inside = std::fabs(i - fx) <= 1 && std::fabs(j - fy) <= 1 && std::fabs(k - fz) <= 1;
                if (d > radius_km && !inside) continue;
                if (n < cap) {
                    idx_out[n] = idx;
                    t_out[n] = origin_time + d * 0.5 * (s_src + slowness[idx]);
                }
                n++;
            }
    return n;
}

// The self-test gate's host solver: SphericalEikonal.Relax (SphericalEikonal.cs:284-325) for
// uniform grids, the reference's settle tolerance and round cap.
std::vector<double> relax_for_selftest(const Grid& g, const double* slowness, const std::vector<int32_t>& seed_idx,
                                       const std::vector<double>& seed_t);

// The LSQR self-test gate's host solver: Lsqr.Solve (Numerics/Lsqr.cs:33-152), sequential sums.
// Returns the iteration count and writes x[n].
int lsqr_for_selftest(int m, int n, const int32_t* row_ptr, const int32_t* col, const double* val, const double* b,
                      double damp, int max_it, double atol, double btol, double conlim, double* x);

}  // namespace host
}  // namespace ts
