// Device geometry for the ray tracer: GeoMath (Geo/GeoMath.cs:49-80, 146-151), SphericalGrid
// fractional coordinates and trilinear weights (Geo/SphericalGrid.cs:179-224), and the float32
// travel-time table's Time and Gradient (Forward/TravelTimeTable.cs:116-157), in double with the
// reference's expression order.
#pragma once

#include "ts_common.cuh"

namespace ts {
namespace geo {

struct V3 {
    double x, y, z;
};
TS_DEVINL V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
TS_DEVINL V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
TS_DEVINL V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
TS_DEVINL double norm(V3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

struct GeoPt {
    double lon, lat, dep;
};

// GeoMath.ToCartesian.
TS_DEVINL V3 to_cartesian(double lon_deg, double lat_deg, double depth_km) {
    double r = kEarthRadiusKm - depth_km;
    double sl, cl, so, co;
    sincos(lat_deg * kDeg2Rad, &sl, &cl);
    sincos(lon_deg * kDeg2Rad, &so, &co);
    return {r * cl * co, r * cl * so, r * sl};
}

// GeoMath.FromCartesian.
TS_DEVINL GeoPt from_cartesian(V3 v) {
    double r = norm(v);
    if (r <= 0) return {0, 0, kEarthRadiusKm};
    double z = fmin(fmax(v.z / r, -1.0), 1.0);
    return {atan2(v.y, v.x) * kRad2Deg, asin(z) * kRad2Deg, kEarthRadiusKm - r};
}

// GeoMath.UnwrapLon.
TS_DEVINL double unwrap_lon(double lon, double ref) {
    if (lon < ref - 180) lon += 360 * ceil((ref - 180 - lon) / 360);
    else if (lon > ref + 180) lon -= 360 * ceil((lon - ref - 180) / 360);
    return lon;
}

// A uniform spherical grid as the tracer needs it (GridDefinition + SphericalGrid fields).
struct RGrid {
    int nx, ny, nz, pad;
    double min_lon, min_lat, min_dep;
    double dlon, dlat, ddep;          // degrees, degrees, km
    double dlon_rad, dlat_rad;
    double centre_lon;
    double lon_last, lat_last, dep_last;  // LonDeg[^1], LatDeg[^1], DepthKm[^1]
    double min_spacing_km;            // MinSpacingKm
};

// SphericalGrid.Fractional.
TS_DEVINL void fractional(const RGrid& g, double lon, double lat, double dep, double& fx, double& fy, double& fz) {
    if (lon < g.centre_lon - 180 || lon > g.centre_lon + 180) lon = unwrap_lon(lon, g.centre_lon);
    fx = (lon - g.min_lon) / g.dlon;
    fy = (lat - g.min_lat) / g.dlat;
    fz = (dep - g.min_dep) / g.ddep;
}

// SphericalGrid.TrilinearWeightsFractional: base corner and the eight weights (di fastest).
TS_DEVINL void weights(const RGrid& g, double fx, double fy, double fz, int& i0, int& j0, int& k0, double* w) {
    fx = fmin(fmax(fx, 0.0), double(g.nx - 1));
    fy = fmin(fmax(fy, 0.0), double(g.ny - 1));
    fz = fmin(fmax(fz, 0.0), double(g.nz - 1));
    i0 = min(int(fx), g.nx - 2);
    j0 = min(int(fy), g.ny - 2);
    k0 = min(int(fz), g.nz - 2);
    double tx = fx - i0, ty = fy - j0, tz = fz - k0;
    int n = 0;
#pragma unroll
    for (int dk = 0; dk < 2; dk++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++)
#pragma unroll
            for (int di = 0; di < 2; di++) {
                w[n] = (di == 0 ? 1 - tx : tx) * (dj == 0 ? 1 - ty : ty) * (dk == 0 ? 1 - tz : tz);
                n++;
            }
}

// TravelTimeTable.TimeFractional: trilinear on float32 nodes; +inf if a weighted corner is not finite.
TS_DEVINL double time_fractional(const RGrid& g, const float* __restrict__ tb, double fx, double fy, double fz) {
    int i0, j0, k0;
    double w[8];
    weights(g, fx, fy, fz, i0, j0, k0, w);
    const int64_t nxy = int64_t(g.nx) * g.ny;
    const int64_t base = k0 * nxy + int64_t(j0) * g.nx + i0;
    double t = 0;
    int n = 0;
#pragma unroll
    for (int dk = 0; dk < 2; dk++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++)
#pragma unroll
            for (int di = 0; di < 2; di++) {
                if (w[n] != 0) {
                    float v = __ldg(&tb[base + dk * nxy + dj * g.nx + di]);
                    if (!isfinite(v)) return dinf();
                    t += double(v) * w[n];
                }
                n++;
            }
    return t;
}

TS_DEVINL double table_time(const RGrid& g, const float* tb, double lon, double lat, double dep) {
    double fx, fy, fz;
    fractional(g, lon, lat, dep, fx, fy, fz);
    return time_fractional(g, tb, fx, fy, fz);
}

// TravelTimeTable.Gradient: central differences of the interpolant half a node each side, in
// (east, north, down) s/km.
TS_DEVINL void table_gradient(const RGrid& g, const float* tb, double lon, double lat, double dep, double& ge,
                              double& gn, double& gz) {
    double fx, fy, fz;
    fractional(g, lon, lat, dep, fx, fy, fz);
    const double d = 0.5;
    double tx = (time_fractional(g, tb, fx + d, fy, fz) - time_fractional(g, tb, fx - d, fy, fz)) / (2 * d);
    double ty = (time_fractional(g, tb, fx, fy + d, fz) - time_fractional(g, tb, fx, fy - d, fz)) / (2 * d);
    double tz = (time_fractional(g, tb, fx, fy, fz + d) - time_fractional(g, tb, fx, fy, fz - d)) / (2 * d);
    double r = kEarthRadiusKm - dep;
    double hx = r * cos(lat * kDeg2Rad) * g.dlon_rad;
    double hy = r * g.dlat_rad;
    double hz = g.ddep;
    ge = tx / hx;
    gn = ty / hy;
    gz = tz / hz;
}

// ---- the same Time and Gradient with every corner load issued before any is used ----------------
//
// time_fractional above loads a corner only where its weight is non-zero and stops at the first
// non-finite one, so each load waits on the previous one's test. The forms below compute the base
// corner first, load all eight corners of every evaluation (they lie on the grid: the base is
// clamped to n − 2 on each axis), and then sum in the reference's order with the same skips and the
// same +inf rule: the same values, with the loads of one step in flight together.

// Base corner of the evaluation at (fx, fy, fz) (clamped as weights() clamps).
TS_DEVINL int64_t corner_base(const RGrid& g, double fx, double fy, double fz) {
    fx = fmin(fmax(fx, 0.0), double(g.nx - 1));
    fy = fmin(fmax(fy, 0.0), double(g.ny - 1));
    fz = fmin(fmax(fz, 0.0), double(g.nz - 1));
    const int i0 = min(int(fx), g.nx - 2), j0 = min(int(fy), g.ny - 2), k0 = min(int(fz), g.nz - 2);
    return int64_t(k0) * g.nx * g.ny + int64_t(j0) * g.nx + i0;
}

TS_DEVINL void load_corners(const RGrid& g, const float* __restrict__ tb, int64_t base, float* v) {
    const int64_t nxy = int64_t(g.nx) * g.ny;
#pragma unroll
    for (int n = 0; n < 8; n++) v[n] = __ldg(&tb[base + (n >> 2) * nxy + ((n >> 1) & 1) * g.nx + (n & 1)]);
}

// TimeFractional from loaded corners.
TS_DEVINL double sum_corners(const RGrid& g, double fx, double fy, double fz, const float* v) {
    int i0, j0, k0;
    double w[8];
    weights(g, fx, fy, fz, i0, j0, k0, w);
    double t = 0;
#pragma unroll
    for (int n = 0; n < 8; n++) {
        if (w[n] != 0) {
            if (!isfinite(v[n])) return dinf();
            t += double(v[n]) * w[n];
        }
    }
    return t;
}

TS_DEVINL double table_time_b(const RGrid& g, const float* tb, double lon, double lat, double dep) {
    double fx, fy, fz;
    fractional(g, lon, lat, dep, fx, fy, fz);
    float v[8];
    load_corners(g, tb, corner_base(g, fx, fy, fz), v);
    return sum_corners(g, fx, fy, fz, v);
}

// Gradient: the six evaluations' 48 corners loaded together.
TS_DEVINL void table_gradient_b(const RGrid& g, const float* tb, double lon, double lat, double dep, double& ge,
                                double& gn, double& gz) {
    double fx, fy, fz;
    fractional(g, lon, lat, dep, fx, fy, fz);
    const double d = 0.5;
    float v[6][8];
#pragma unroll
    for (int e = 0; e < 6; e++) {
        const double ex = e == 0 ? fx + d : e == 1 ? fx - d : fx;
        const double ey = e == 2 ? fy + d : e == 3 ? fy - d : fy;
        const double ez = e == 4 ? fz + d : e == 5 ? fz - d : fz;
        load_corners(g, tb, corner_base(g, ex, ey, ez), v[e]);
    }
    const double tx = (sum_corners(g, fx + d, fy, fz, v[0]) - sum_corners(g, fx - d, fy, fz, v[1])) / (2 * d);
    const double ty = (sum_corners(g, fx, fy + d, fz, v[2]) - sum_corners(g, fx, fy - d, fz, v[3])) / (2 * d);
    const double tz = (sum_corners(g, fx, fy, fz + d, v[4]) - sum_corners(g, fx, fy, fz - d, v[5])) / (2 * d);
    double r = kEarthRadiusKm - dep;
    double hx = r * cos(lat * kDeg2Rad) * g.dlon_rad;
    double hy = r * g.dlat_rad;
    double hz = g.ddep;
    ge = tx / hx;
    gn = ty / hy;
    gz = tz / hz;
}

// ---- the same Time and Gradient computed by one warp for one point ------------------------------
//
// For a ray traced by a whole warp: the lanes load the corners (lane l loads corner l & 7 of
// evaluation l >> 3, and of evaluation 4 + ((l >> 3) & 1) in a second load), each of the six
// gradient evaluations is summed in its own lane, and every lane then takes the six sums by shuffles
// and forms the gradient. Every value is computed with the operations and in the order of the forms
// above, so both give the same bits. All 32 lanes must call these together.

TS_DEVINL int64_t corner_offset(const RGrid& g, int n) {
    return (n >> 2) * (int64_t(g.nx) * g.ny) + ((n >> 1) & 1) * g.nx + (n & 1);
}

TS_DEVINL double table_time_w(const RGrid& g, const float* tb, double lon, double lat, double dep, int lane) {
    double fx, fy, fz;
    fractional(g, lon, lat, dep, fx, fy, fz);
    const float mine = __ldg(&tb[corner_base(g, fx, fy, fz) + corner_offset(g, lane & 7)]);
    float v[8];
#pragma unroll
    for (int n = 0; n < 8; n++) v[n] = __shfl_sync(0xffffffffu, mine, n);
    return sum_corners(g, fx, fy, fz, v);
}

TS_DEVINL void table_gradient_w(const RGrid& g, const float* tb, double lon, double lat, double dep, double& ge,
                                double& gn, double& gz, int lane) {
    double fx, fy, fz;
    fractional(g, lon, lat, dep, fx, fy, fz);
    const double d = 0.5;
    auto at = [&](int e, double& ex, double& ey, double& ez) {
        ex = e == 0 ? fx + d : e == 1 ? fx - d : fx;
        ey = e == 2 ? fy + d : e == 3 ? fy - d : fy;
        ez = e == 4 ? fz + d : e == 5 ? fz - d : fz;
    };
    const int n = lane & 7;
    double ax, ay, az, bx, by, bz;
    at(lane >> 3, ax, ay, az);
    at(4 + ((lane >> 3) & 1), bx, by, bz);
    const float va = __ldg(&tb[corner_base(g, ax, ay, az) + corner_offset(g, n)]);
    const float vb = __ldg(&tb[corner_base(g, bx, by, bz) + corner_offset(g, n)]);
    const int me = lane < 6 ? lane : 0;  // the evaluation this lane sums
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const float x = __shfl_sync(0xffffffffu, va, 8 * (me & 3) + k);
        const float y = __shfl_sync(0xffffffffu, vb, 8 * (me & 1) + k);
        v[k] = me < 4 ? x : y;
    }
    double ex, ey, ez;
    at(me, ex, ey, ez);
    const double te = sum_corners(g, ex, ey, ez, v);
    double t[6];
#pragma unroll
    for (int e = 0; e < 6; e++) t[e] = __shfl_sync(0xffffffffu, te, e);
    const double tx = (t[0] - t[1]) / (2 * d);
    const double ty = (t[2] - t[3]) / (2 * d);
    const double tz = (t[4] - t[5]) / (2 * d);
    double r = kEarthRadiusKm - dep;
    double hx = r * cos(lat * kDeg2Rad) * g.dlon_rad;
    double hy = r * g.dlat_rad;
    double hz = g.ddep;
    ge = tx / hx;
    gn = ty / hy;
    gz = tz / hz;
}

// SphericalGrid.Contains (Geo/SphericalGrid.cs:186-192).
TS_DEVINL bool contains(const RGrid& g, double lon, double lat, double dep, double tol) {
    double fx, fy, fz;
    fractional(g, lon, lat, dep, fx, fy, fz);
    return fx >= -tol && fx <= g.nx - 1 + tol && fy >= -tol && fy <= g.ny - 1 + tol && fz >= -tol && fz <= g.nz - 1 + tol;
}

// VelocityModel1D.Evaluate (Model/VelocityModel1D.cs:31-45): piecewise linear in depth, the upper
// value on an interface, the first node's value above it and the last node's below the last.
TS_HDINL double background_1d(const double* depth, const double* v, int n, double d) {
    if (d <= depth[0]) return v[0];
    for (int i = 1; i < n; i++) {
        if (d > depth[i]) continue;
        if (depth[i] - depth[i - 1] <= 1e-12) continue;  // discontinuity: move below it
        const double t = (d - depth[i - 1]) / (depth[i] - depth[i - 1]);
        return v[i - 1] + t * (v[i] - v[i - 1]);
    }
    return v[n - 1];
}

}  // namespace geo
}  // namespace ts
