// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of TomoSTAR's forward path and of its callers on either side (LSQR, event
// location, the forward domain and model), used by the tests, by the smoke check and by bench.py's
// CPU-baseline legs as the checker and baseline. The product (tomostar_b200/) never links, loads or
// calls this file.
//
// Parity status: the reference is C# (.NET 10) and cannot be built or run here, so no bitwise
// reference output exists. The forward path is pinned by the reference's own known-answer tests
// (tests/TomoStar.Tests/NumericsTests.cs:88-123) and the analytic cases of its validation exporter
// (validation/TomoStar.Validation/Program.cs:107-143); LSQR by SciPy's lsqr (the SOL kernel
// Lsqr.cs follows); location by PipelineTests.RelocationMovesEventsTowardsTheTruth
// (tests/TomoStar.Tests/PipelineTests.cs:95-107) and hand-worked medians and gaps; the forward
// domain and the 1-D background by hand-worked cases. tests/test_oracle.py and tests/test_domain.py
// run them.
//
// Every function cites the reference lines it follows. Arithmetic is kept in the reference's
// expression order and the file is compiled with -ffp-contract=off, so a double result is the
// one .NET computes on the same libm (glibc on Linux).
//
// Extension not in the reference: a grid may carry an explicit depth array (variable, e.g.
// geometric, vertical spacing). The z-axis spacing of the upwind update is then the distance
// to the neighbour actually used, and the second-order term uses the non-uniform one-sided
// three-point derivative. With a uniform grid the reference arithmetic is used unchanged.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <atomic>
#include <vector>

namespace {

constexpr double kEarthRadiusKm = 6371.0;            // Geo/GeoMath.cs:43
constexpr double kDeg2Rad = M_PI / 180.0;            // Geo/GeoMath.cs:45
constexpr double kRad2Deg = 180.0 / M_PI;            // Geo/GeoMath.cs:46
constexpr double kInf = std::numeric_limits<double>::infinity();

struct V3 {
    double x, y, z;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double norm(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }  // GeoMath.cs:18

// GeoMath.ToCartesian (Geo/GeoMath.cs:49-56).
inline V3 to_cartesian(double lon_deg, double lat_deg, double depth_km) {
    double r = kEarthRadiusKm - depth_km;
    double lat = lat_deg * kDeg2Rad;
    double lon = lon_deg * kDeg2Rad;
    double cl = std::cos(lat);
    return {r * cl * std::cos(lon), r * cl * std::sin(lon), r * std::sin(lat)};
}

struct Geo {
    double lon, lat, depth;
};

// GeoMath.FromCartesian (Geo/GeoMath.cs:61-68).
inline Geo from_cartesian(V3 v) {
    double r = norm(v);
    if (r <= 0) return {0, 0, kEarthRadiusKm};
    double lat = std::asin(std::clamp(v.z / r, -1.0, 1.0)) * kRad2Deg;
    double lon = std::atan2(v.y, v.x) * kRad2Deg;
    return {lon, lat, kEarthRadiusKm - r};
}

// GeoMath.LocalFrame (Geo/GeoMath.cs:71-80).
inline void local_frame(double lon_deg, double lat_deg, V3& east, V3& north, V3& up) {
    double lat = lat_deg * kDeg2Rad;
    double lon = lon_deg * kDeg2Rad;
    double sl = std::sin(lat), cl = std::cos(lat), so = std::sin(lon), co = std::cos(lon);
    east = {-so, co, 0};
    north = {-sl * co, -sl * so, cl};
    up = {cl * co, cl * so, sl};
}

// GeoMath.UnwrapLon (Geo/GeoMath.cs:146-151).
inline double unwrap_lon(double lon, double ref) {
    if (lon < ref - 180) lon += 360 * std::ceil((ref - 180 - lon) / 360);
    else if (lon > ref + 180) lon -= 360 * std::ceil((lon - ref - 180) / 360);
    return lon;
}

}  // namespace

extern "C" {

// GridDefinition (Geo/SphericalGrid.cs:13-31) plus the optional depth array of the extension.
struct or_grid_def {
    double min_lon, max_lon, min_lat, max_lat, min_depth_km, max_depth_km;
    int32_t nx, ny, nz, _pad;
    const double* depth_km;  // nz depths (variable vertical spacing) or null (uniform)
};

}  // extern "C"

namespace {

// SphericalGrid (Geo/SphericalGrid.cs:84-116).
struct Grid {
    int nx, ny, nz;
    double min_lon, min_lat, min_dep;
    double dlon, dlat, ddep;  // GridDefinition.DLon/DLat/DDepth (SphericalGrid.cs:28-30)
    double centre_lon, dlon_rad, dlat_rad, ddep_km;
    bool variable;
    std::vector<double> lon, lat, coslat, dep, rad;

    explicit Grid(const or_grid_def& d) {
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
        ddep_km = ddep;
    }
    int count() const { return nx * ny * nz; }
    int index(int i, int j, int k) const { return (k * ny + j) * nx + i; }  // SphericalGrid.cs:135
    V3 cartesian(int i, int j, int k) const { return to_cartesian(lon[i], lat[j], dep[k]); }

    // Fractional depth index; the extension inverts the depth array piecewise linearly.
    double frac_z(double depth_km) const {
        if (!variable) return (depth_km - min_dep) / ddep;
        if (depth_km <= dep[0]) return (depth_km - dep[0]) / (dep[1] - dep[0]);
        if (depth_km >= dep[nz - 1]) return (nz - 1) + (depth_km - dep[nz - 1]) / (dep[nz - 1] - dep[nz - 2]);
        int k = int(std::upper_bound(dep.begin(), dep.end(), depth_km) - dep.begin()) - 1;
        return k + (depth_km - dep[k]) / (dep[k + 1] - dep[k]);
    }
    // SphericalGrid.Fractional (SphericalGrid.cs:179-184).
    void fractional(double lon_deg, double lat_deg, double depth_km, double& fx, double& fy, double& fz) const {
        if (lon_deg < centre_lon - 180 || lon_deg > centre_lon + 180) lon_deg = unwrap_lon(lon_deg, centre_lon);
        fx = (lon_deg - min_lon) / dlon;
        fy = (lat_deg - min_lat) / dlat;
        fz = frac_z(depth_km);
    }
    // SphericalGrid.TrilinearWeightsFractional (SphericalGrid.cs:205-224).
    void weights_fractional(double fx, double fy, double fz, int* nodes, double* w) const {
        fx = std::clamp(fx, 0.0, double(nx - 1));
        fy = std::clamp(fy, 0.0, double(ny - 1));
        fz = std::clamp(fz, 0.0, double(nz - 1));
        int i0 = std::min(int(fx), nx - 2), j0 = std::min(int(fy), ny - 2), k0 = std::min(int(fz), nz - 2);
        double tx = fx - i0, ty = fy - j0, tz = fz - k0;
        int n = 0;
        for (int dk = 0; dk < 2; dk++)
            for (int dj = 0; dj < 2; dj++)
                for (int di = 0; di < 2; di++) {
                    nodes[n] = index(i0 + di, j0 + dj, k0 + dk);
                    w[n] = (di == 0 ? 1 - tx : tx) * (dj == 0 ? 1 - ty : ty) * (dk == 0 ? 1 - tz : tz);
                    n++;
                }
    }
    void weights(double lon_deg, double lat_deg, double depth_km, int* nodes, double* w) const {
        double fx, fy, fz;
        fractional(lon_deg, lat_deg, depth_km, fx, fy, fz);
        weights_fractional(fx, fy, fz, nodes, w);
    }
    // SphericalGrid.Interpolate (SphericalGrid.cs:227-235).
    double interpolate(const double* field, double lon_deg, double lat_deg, double depth_km) const {
        int nodes[8];
        double w[8];
        weights(lon_deg, lat_deg, depth_km, nodes, w);
        double sum = 0;
        for (int n = 0; n < 8; n++) sum += field[nodes[n]] * w[n];
        return sum;
    }
    // SphericalGrid.MinSpacingKm (SphericalGrid.cs:159-164).
    double min_spacing_km() const {
        double r_min = rad[nz - 1];
        double cos_min = *std::min_element(coslat.begin(), coslat.end());
        double dz = ddep_km;
        if (variable) {
            dz = kInf;
            for (int k = 0; k + 1 < nz; k++) dz = std::min(dz, dep[k + 1] - dep[k]);
        }
        return std::min(dz, std::min(r_min * dlat_rad, r_min * cos_min * dlon_rad));
    }
};

// GridMetric (Forward/SphericalEikonal.cs:15-35), with the z spacing per interval for the extension.
struct Metric {
    const Grid& g;
    std::vector<double> hlon, hlat, dz;  // dz[k] = depth[k+1] - depth[k] (extension only)
    double hr;
    explicit Metric(const Grid& grid) : g(grid) {
        hlon.resize(size_t(g.ny) * g.nz);
        hlat.resize(g.nz);
        for (int k = 0; k < g.nz; k++) {
            hlat[k] = g.rad[k] * g.dlat_rad;
            for (int j = 0; j < g.ny; j++) hlon[size_t(k) * g.ny + j] = std::max(1e-9, g.rad[k] * g.coslat[j] * g.dlon_rad);
        }
        hr = g.ddep_km;
        if (g.variable) {
            dz.resize(g.nz - 1);
            for (int k = 0; k + 1 < g.nz; k++) dz[k] = g.dep[k + 1] - g.dep[k];
        }
    }
};

// One upwind term: effective time, effective spacing, the neighbour's own time.
struct Term {
    double t, h, n;
};

// Stable insertion sort by effective time (SphericalEikonal.cs:262-275).
inline void sort_terms(Term* q, int used) {
    for (int a = 1; a < used; a++) {
        Term x = q[a];
        int b = a - 1;
        while (b >= 0 && q[b].t > x.t) { q[b + 1] = q[b]; b--; }
        q[b + 1] = x;
    }
}

// The Godunov root over the used terms, largest subset first (SphericalEikonal.cs:179-199, 364-379).
inline double godunov(const Term* q, int used, double s) {
    for (int terms = used; terms >= 1; terms--) {
        double sw = 0, swt = 0, swt2 = 0;
        for (int r = 0; r < terms; r++) {
            double w = 1.0 / (q[r].h * q[r].h);
            sw += w;
            swt += w * q[r].t;
            swt2 += w * q[r].t * q[r].t;
        }
        double disc = swt * swt - sw * (swt2 - s * s);
        if (disc < 0) continue;
        double root = (swt + std::sqrt(disc)) / sw;
        bool ok = true;
        for (int r = 0; r < terms; r++)
            if (root < q[r].n) { ok = false; break; }
        if (ok) return root;
    }
    return kInf;
}

// Uniform-axis term (SphericalEikonal.cs:381-395 / EikonalOpenCl.cs:432-450): pick the smaller
// neighbour, promote to second order when its partner beyond is finite and not larger.
inline void axis_term(double minus, double plus, double minus2, double plus2, double h, bool second_order, Term* q,
                      int& used) {
    double first, t2;
    if (minus <= plus) { first = minus; t2 = minus2; }
    else { first = plus; t2 = plus2; }
    if (!std::isfinite(first)) return;
    if (!second_order) t2 = kInf;
    if (std::isfinite(t2) && t2 <= first) q[used] = {(4 * first - t2) / 3, 2 * h / 3, first};
    else q[used] = {first, h, first};
    used++;
}

// Extension: z-axis term on a non-uniform axis. h1 = spacing to the first neighbour, h2 = from
// there to the second. The one-sided derivative a·T0 + b·T1 + c·T2 with a = (2h1+h2)/(h1(h1+h2)),
// b = −(h1+h2)/(h1 h2), c = h1/(h2(h1+h2)) is written as (T0 − te)/he: he = 1/a, te = −(b T1 + c T2)/a.
inline void axis_term_var(double minus, double plus, double minus2, double plus2, double hm, double hp, double hm2,
                          double hp2, bool second_order, Term* q, int& used) {
    double first, t2, h1, h2;
    if (minus <= plus) { first = minus; t2 = minus2; h1 = hm; h2 = hm2; }
    else { first = plus; t2 = plus2; h1 = hp; h2 = hp2; }
    if (!std::isfinite(first)) return;
    if (!second_order) t2 = kInf;
    if (std::isfinite(t2) && t2 <= first) {
        double a = (2 * h1 + h2) / (h1 * (h1 + h2));
        double b = (h1 + h2) / (h1 * h2);
        double c = h1 / (h2 * (h1 + h2));
        q[used] = {(b * first - c * t2) / a, 1 / a, first};
    } else {
        q[used] = {first, h1, first};
    }
    used++;
}

// RelaxNode (SphericalEikonal.cs:349-396): the upwind update of one node from the field values.
inline double relax_node(const Metric& m, const double* s_arr, const double* f, int idx, int i, int j, int k,
                         bool second_order) {
    const Grid& g = m.g;
    double s = s_arr[idx];
    if (!(s > 0)) return kInf;
    int nx = g.nx, ny = g.ny, nz = g.nz, nxy = nx * ny;
    Term q[3];
    int used = 0;
    auto at = [&](bool ok, int off) { return ok ? f[idx + off] : kInf; };
    axis_term(at(i > 0, -1), at(i + 1 < nx, 1), at(i > 1, -2), at(i + 2 < nx, 2), m.hlon[size_t(k) * ny + j],
              second_order, q, used);
    axis_term(at(j > 0, -nx), at(j + 1 < ny, nx), at(j > 1, -2 * nx), at(j + 2 < ny, 2 * nx), m.hlat[k], second_order,
              q, used);
    if (!g.variable) {
        axis_term(at(k > 0, -nxy), at(k + 1 < nz, nxy), at(k > 1, -2 * nxy), at(k + 2 < nz, 2 * nxy), m.hr,
                  second_order, q, used);
    } else {
        double hm = k > 0 ? m.dz[k - 1] : 1, hp = k + 1 < nz ? m.dz[k] : 1;
        double hm2 = k > 1 ? m.dz[k - 2] : 1, hp2 = k + 2 < nz ? m.dz[k + 1] : 1;
        axis_term_var(at(k > 0, -nxy), at(k + 1 < nz, nxy), at(k > 1, -2 * nxy), at(k + 2 < nz, 2 * nxy), hm, hp, hm2,
                      hp2, second_order, q, used);
    }
    if (used == 0) return kInf;
    sort_terms(q, used);
    return godunov(q, used, s);
}

// SphericalEikonal.PlaneBounds (SphericalEikonal.cs:341-347).
inline void plane_bounds(int nx, int ny, int nz, int p, int& i0, int& i1, int& k0, int& k1) {
    i0 = std::max(0, p - (ny - 1) - (nz - 1));
    i1 = std::min(nx - 1, p);
    k0 = std::max(0, p - (nx - 1) - (ny - 1));
    k1 = std::min(nz - 1, p);
}

// SphericalEikonal.SweepRoundCap (SphericalEikonal.cs:335).
inline int sweep_round_cap(const Grid& g) { return std::max(32, (g.nx + g.ny + g.nz) / 4); }

// FrontHeap (SphericalEikonal.cs:404-475): 4-ary min-heap, one entry per node, decrease-key in place.
struct FrontHeap {
    struct Entry {
        double key;
        int node;
    };
    std::vector<Entry> e;
    std::vector<int> at;  // slot + 1; 0 = absent
    int count = 0;
    FrontHeap(int nodes, int capacity) : e(capacity), at(nodes, 0) {}
    void set(int node, double key) {
        int i = at[node] - 1;
        if (i < 0) {
            if (count == int(e.size())) e.resize(size_t(count) * 2);
            i = count++;
        }
        while (i > 0) {
            int p = (i - 1) >> 2;
            if (e[p].key <= key) break;
            e[i] = e[p];
            at[e[i].node] = i + 1;
            i = p;
        }
        e[i] = {key, node};
        at[node] = i + 1;
    }
    bool pop(int& node) {
        if (count == 0) { node = -1; return false; }
        node = e[0].node;
        at[node] = 0;
        Entry last = e[--count];
        if (count == 0) return true;
        int i = 0;
        for (;;) {
            int c = 4 * i + 1;
            if (c >= count) break;
            int best = c;
            double best_key = e[c].key;
            int end = std::min(c + 4, count);
            for (int q = c + 1; q < end; q++)
                if (e[q].key < best_key) { best = q; best_key = e[q].key; }
            if (best_key >= last.key) break;
            e[i] = e[best];
            at[e[i].node] = i + 1;
            i = best;
        }
        e[i] = last;
        at[last.node] = i + 1;
        return true;
    }
};

// TravelTimeTable float32 storage (Forward/TravelTimeTable.cs:73) and trilinear time (:122-136).
struct Table {
    const Grid& g;
    const float* v;
    double src_lon, src_lat, src_dep;
    double time_fractional(double fx, double fy, double fz) const {
        int nodes[8];
        double w[8];
        g.weights_fractional(fx, fy, fz, nodes, w);
        double t = 0;
        for (int n = 0; n < 8; n++) {
            if (w[n] == 0) continue;
            float x = v[nodes[n]];
            if (!std::isfinite(x)) return kInf;
            t += x * w[n];
        }
        return t;
    }
    double time(double lon, double lat, double dep) const {
        double fx, fy, fz;
        g.fractional(lon, lat, dep, fx, fy, fz);
        return time_fractional(fx, fy, fz);
    }
    // TravelTimeTable.Gradient (TravelTimeTable.cs:143-157): central differences of the interpolant,
    // half a node each side, in (east, north, down) s/km.
    void gradient(double lon, double lat, double dep, double& ge, double& gn, double& gz) const {
        double fx, fy, fz;
        g.fractional(lon, lat, dep, fx, fy, fz);
        const double d = 0.5;
        double tx = (time_fractional(fx + d, fy, fz) - time_fractional(fx - d, fy, fz)) / (2 * d);
        double ty = (time_fractional(fx, fy + d, fz) - time_fractional(fx, fy - d, fz)) / (2 * d);
        double tz = (time_fractional(fx, fy, fz + d) - time_fractional(fx, fy, fz - d)) / (2 * d);
        double r = kEarthRadiusKm - dep;
        double hx = r * std::cos(lat * kDeg2Rad) * g.dlon_rad;
        double hy = r * g.dlat_rad;
        double hz = g.ddep_km;
        ge = tx / hx; gn = ty / hy; gz = tz / hz;
    }
};

// RayTracing.Backtrack (Forward/RayTracing.cs:73-111). Returns false where the reference returns null.
bool backtrack(const Table& tb, double lon, double lat, double dep, double step_km, std::vector<Geo>& path) {
    const Grid& g = tb.g;
    double st_dep = std::clamp(tb.src_dep, g.dep[0], g.dep[g.nz - 1]);
    V3 station = to_cartesian(tb.src_lon, tb.src_lat, st_dep);
    V3 p = to_cartesian(lon, lat, dep);
    path.clear();
    path.push_back({lon, lat, dep});
    double t0 = tb.time(lon, lat, dep);
    if (!std::isfinite(t0)) return false;
    int max_steps = 20 * int(std::ceil(norm(sub(p, station)) / step_km + 10));
    double last_t = t0;
    int stalls = 0;
    for (int step = 0; step < max_steps; step++) {
        if (norm(sub(p, station)) <= 1.5 * step_km) break;
        Geo gp = from_cartesian(p);
        double ge, gn, gz;
        tb.gradient(gp.lon, gp.lat, gp.depth, ge, gn, gz);
        if (!std::isfinite(ge) || !std::isfinite(gn) || !std::isfinite(gz)) return false;
        V3 e, nn, up;
        local_frame(gp.lon, gp.lat, e, nn, up);
        V3 grad = add(add(scale(e, ge), scale(nn, gn)), scale(up, -gz));
        double nrm = norm(grad);
        if (nrm < 1e-12) return false;
        p = sub(p, scale(grad, step_km / nrm));
        Geo q = from_cartesian(p);
        q = {std::clamp(unwrap_lon(q.lon, g.centre_lon), g.lon[0], g.lon[g.nx - 1]),
             std::clamp(q.lat, g.lat[0], g.lat[g.ny - 1]), std::clamp(q.depth, g.dep[0], g.dep[g.nz - 1])};
        p = to_cartesian(q.lon, q.lat, q.depth);
        path.push_back(q);
        double t = tb.time(q.lon, q.lat, q.depth);
        if (!(t < last_t)) {
            if (++stalls > 20) return false;
        } else {
            stalls = 0;
        }
        last_t = std::min(last_t, t);
    }
    path.push_back({tb.src_lon, tb.src_lat, st_dep});
    return true;
}

double evaluate_1d(const double* depth, const double* v, int n, double d);
bool grid_contains(const Grid& g, double lon, double lat, double dep, double tol);

// RayTracing.Kernel (RayTracing.cs:126-159): (node, length) in first-visit order, each length summed
// in visit order like the reference's dictionary. With a background (nbg > 0), pieces outside the
// inversion grid (tolerance 1e-6) are not attributed: their length times the background's slowness
// 1/v(depth) is summed into *outside instead.
void ray_kernel(const Grid& inv, const std::vector<Geo>& ray, std::vector<int>& keys, std::vector<double>& vals,
                int nbg = 0, const double* bgd = nullptr, const double* bgv = nullptr, double* outside = nullptr) {
    if (outside) *outside = 0;
    keys.clear();
    vals.clear();
    // node -> slot of keys/vals: open addressing with linear probing, kept under half full
    size_t cap = 1024;
    std::vector<int> hk(cap, -1), hv(cap, -1);
    auto find = [&](int node) -> int {
        size_t m = cap - 1, h = (uint32_t(node) * 2654435761u) & m;
        while (hk[h] != -1 && hk[h] != node) h = (h + 1) & m;
        if (hk[h] == node) return hv[h];
        return -1 - int(h);
    };
    auto insert_new = [&](int node, double v) {
        if (keys.size() * 2 >= cap) {
            cap *= 2;
            hk.assign(cap, -1); hv.assign(cap, -1);
            for (size_t s = 0; s < keys.size(); s++) {
                size_t m = cap - 1, h = (uint32_t(keys[s]) * 2654435761u) & m;
                while (hk[h] != -1) h = (h + 1) & m;
                hk[h] = keys[s]; hv[h] = int(s);
            }
        }
        size_t m = cap - 1, h = (uint32_t(node) * 2654435761u) & m;
        while (hk[h] != -1) h = (h + 1) & m;
        hk[h] = node; hv[h] = int(keys.size());
        keys.push_back(node);
        vals.push_back(v);
    };
    double h = 0.5 * inv.min_spacing_km();
    int nodes[8];
    double w[8];
    for (size_t i = 1; i < ray.size(); i++) {
        V3 a = to_cartesian(ray[i - 1].lon, ray[i - 1].lat, ray[i - 1].depth);
        V3 b = to_cartesian(ray[i].lon, ray[i].lat, ray[i].depth);
        double len = norm(sub(b, a));
        if (len <= 0) continue;
        int pieces = std::max(1, int(std::ceil(len / h)));
        double dl = len / pieces;
        for (int q = 0; q < pieces; q++) {
            Geo mid = from_cartesian(add(a, scale(sub(b, a), (q + 0.5) / pieces)));
            if (nbg > 0 && !grid_contains(inv, mid.lon, mid.lat, mid.depth, 1e-6)) {
                *outside += dl * (1 / evaluate_1d(bgd, bgv, nbg, mid.depth));
                continue;
            }
            inv.weights(mid.lon, mid.lat, mid.depth, nodes, w);
            for (int n = 0; n < 8; n++) {
                if (w[n] == 0) continue;
                double v = dl * w[n] * 1.0;
                int s = find(nodes[n]);
                if (s >= 0) vals[s] = vals[s] + v;
                else insert_new(nodes[n], v);
            }
        }
    }
}

}  // namespace

extern "C" {

// ---- geometry --------------------------------------------------------------------------------

// GridMetric arrays (SphericalEikonal.cs:17-29): hlon[ny*nz], hlat[nz], *hr; dz[nz-1] when variable.
void or_metric(const or_grid_def* d, double* hlon, double* hlat, double* hr, double* dz) {
    Grid g(*d);
    Metric m(g);
    std::copy(m.hlon.begin(), m.hlon.end(), hlon);
    std::copy(m.hlat.begin(), m.hlat.end(), hlat);
    *hr = m.hr;
    if (dz && g.variable) std::copy(m.dz.begin(), m.dz.end(), dz);
}

// Node coordinates: lon[nx], lat[ny], coslat[ny], depth[nz] (SphericalGrid.cs:96-111).
void or_grid_coords(const or_grid_def* d, double* lon, double* lat, double* coslat, double* depth) {
    Grid g(*d);
    std::copy(g.lon.begin(), g.lon.end(), lon);
    std::copy(g.lat.begin(), g.lat.end(), lat);
    std::copy(g.coslat.begin(), g.coslat.end(), coslat);
    std::copy(g.dep.begin(), g.dep.end(), depth);
}

double or_min_spacing_km(const or_grid_def* d) { return Grid(*d).min_spacing_km(); }

void or_to_cartesian(double lon, double lat, double dep, double* xyz) {
    V3 v = to_cartesian(lon, lat, dep);
    xyz[0] = v.x; xyz[1] = v.y; xyz[2] = v.z;
}

void or_from_cartesian(const double* xyz, double* geo) {
    Geo g = from_cartesian({xyz[0], xyz[1], xyz[2]});
    geo[0] = g.lon; geo[1] = g.lat; geo[2] = g.depth;
}

// SphericalGrid.TrilinearWeights (SphericalGrid.cs:199-224).
void or_trilinear(const or_grid_def* d, double lon, double lat, double dep, int32_t* nodes, double* w) {
    Grid g(*d);
    int n[8];
    g.weights(lon, lat, dep, n, w);
    for (int q = 0; q < 8; q++) nodes[q] = n[q];
}

double or_interpolate(const or_grid_def* d, const double* field, double lon, double lat, double dep) {
    return Grid(*d).interpolate(field, lon, lat, dep);
}

// ---- seeds -----------------------------------------------------------------------------------

// SphericalEikonal.PointSource (SphericalEikonal.cs:68-100). Returns the seed count (or, when it
// exceeds cap, the count needed, with nothing written past cap).
int32_t or_point_source(const or_grid_def* d, const double* slowness, double lon, double lat, double depth_km,
                        double origin_time, double radius_cells, int32_t* idx_out, double* t_out, int32_t cap) {
    Grid g(*d);
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
    double h_r = g.ddep_km;
    if (g.variable) {  // extension: the local vertical spacing at the source
        int kk = std::min(int(fz), g.nz - 2);
        h_r = g.dep[kk + 1] - g.dep[kk];
    }
    double radius_km = radius_cells * std::max(h_lon, std::max(h_lat, h_r));
    int ri = int(std::ceil(radius_km / h_lon)), rj = int(std::ceil(radius_km / h_lat)), rk = int(std::ceil(radius_km / h_r));
    int i0 = int(std::nearbyint(fx)), j0 = int(std::nearbyint(fy)), k0 = int(std::nearbyint(fz));  // Math.Round: half to even
    if (g.variable) rk += 2;  // extension: vertical spacing varies; the distance test below decides
    int n = 0;
    for (int k = std::max(0, k0 - rk); k <= std::min(g.nz - 1, k0 + rk); k++)
        for (int j = std::max(0, j0 - rj); j <= std::min(g.ny - 1, j0 + rj); j++)
            for (int i = std::max(0, i0 - ri); i <= std::min(g.nx - 1, i0 + ri); i++) {
                int idx = g.index(i, j, k);
                double dd = norm(sub(g.cartesian(i, j, k), src));
                bool inside = std::fabs(i - fx) <= 1 && std::fabs(j - fy) <= 1 && std::fabs(k - fz) <= 1;
                if (dd > radius_km && !inside) continue;
                if (n < cap) {
                    idx_out[n] = idx;
                    t_out[n] = origin_time + dd * 0.5 * (s_src + slowness[idx]);
                }
                n++;
            }
    return n;
}

// ---- solvers ---------------------------------------------------------------------------------

// SphericalEikonal.Relax (SphericalEikonal.cs:284-325), plane-ordered fast sweeping: phase 0 first
// order, phase 1 with second-order promotion; a round is eight sweeps; a phase ends at a round in
// which no node dropped by more than tol (reference: SettleTolerance = 1e-7, :332); tol = 0 runs
// to the exact fixed point. max_rounds <= 0 uses SweepRoundCap (:335). rounds_out[2] receives the
// rounds of each phase. Returns 1 when both phases settled within the cap, else 0.
int32_t or_relax(const or_grid_def* d, const double* slowness, int32_t n_seeds, const int32_t* seed_idx,
                 const double* seed_t, int32_t max_rounds, double tol, double* out, int32_t* rounds_out) {
    Grid g(*d);
    Metric m(g);
    int n = g.count();
    std::fill(out, out + n, kInf);
    std::vector<uint8_t> fixed(n, 0);
    for (int q = 0; q < n_seeds; q++) {
        int s = seed_idx[q];
        if (unsigned(s) >= unsigned(n)) continue;
        out[s] = std::min(out[s], seed_t[q]);
        fixed[s] = 1;
    }
    int nx = g.nx, ny = g.ny, nz = g.nz;
    int cap = max_rounds > 0 ? max_rounds : sweep_round_cap(g);
    int settled_all = 1;
    for (int phase = 0; phase < 2; phase++) {
        int settled = 0, round = 0;
        for (round = 0; round < cap; round++) {
            bool changed = false;
            for (int dir = 0; dir < 8; dir++)
                for (int p = 0; p < nx + ny + nz - 2; p++) {
                    int i0, i1, k0, k1;
                    plane_bounds(nx, ny, nz, p, i0, i1, k0, k1);
                    for (int kp = k0; kp <= k1; kp++)
                        for (int ip = i0; ip <= i1; ip++) {
                            int jp = p - ip - kp;
                            if (jp < 0 || jp >= ny) continue;
                            int i = (dir & 1) ? nx - 1 - ip : ip;
                            int j = (dir & 2) ? ny - 1 - jp : jp;
                            int k = (dir & 4) ? nz - 1 - kp : kp;
                            int idx = g.index(i, j, k);
                            if (fixed[idx]) continue;
                            double cur = out[idx];
                            double cand = relax_node(m, slowness, out, idx, i, j, k, phase == 1);
                            if (!(cand < cur)) continue;
                            out[idx] = cand;
                            if (!std::isfinite(cur) || cur - cand > tol) changed = true;
                        }
                }
            if (!changed) { settled = 1; round++; break; }
        }
        if (rounds_out) rounds_out[phase] = round;
        if (!settled) settled_all = 0;
    }
    return settled_all;
}

// One round of eight sweeps of one field (the body of Relax's round loop); true when a node dropped
// from +inf or by more than tol.
static bool relax_round(const Grid& g, const Metric& m, const double* slowness, double* out,
                        const std::vector<uint8_t>& fixed, int phase, double tol) {
    int nx = g.nx, ny = g.ny, nz = g.nz;
    bool changed = false;
    for (int dir = 0; dir < 8; dir++)
        for (int p = 0; p < nx + ny + nz - 2; p++) {
            int i0, i1, k0, k1;
            plane_bounds(nx, ny, nz, p, i0, i1, k0, k1);
            for (int kp = k0; kp <= k1; kp++)
                for (int ip = i0; ip <= i1; ip++) {
                    int jp = p - ip - kp;
                    if (jp < 0 || jp >= ny) continue;
                    int i = (dir & 1) ? nx - 1 - ip : ip;
                    int j = (dir & 2) ? ny - 1 - jp : jp;
                    int k = (dir & 4) ? nz - 1 - kp : kp;
                    int idx = g.index(i, j, k);
                    if (fixed[idx]) continue;
                    double cur = out[idx];
                    double cand = relax_node(m, slowness, out, idx, i, j, k, phase == 1);
                    if (!(cand < cur)) continue;
                    out[idx] = cand;
                    if (!std::isfinite(cur) || cur - cand > tol) changed = true;
                }
        }
    return changed;
}

// A batch of fields on one slowness as EikonalOpenCl.Sweep solves it (EikonalOpenCl.cs:215-270): one
// `changed` flag for the whole batch, so every field is swept until no field of the batch moved by
// more than tol in a round, and the batch enters phase 1 together. A field that settled early keeps
// being swept, which can move it below tol: its bits may differ from a solve on its own (Relax, and
// the per-field settling of the CUDA engine) by a few ulps. Seeds of field e are
// seed_idx/seed_t[seed_off[e] .. seed_off[e+1]); out is field-major. Returns 1 when settled.
int32_t or_relax_batch(const or_grid_def* d, const double* slowness, int32_t batch, const int32_t* seed_off,
                       const int32_t* seed_idx, const double* seed_t, int32_t max_rounds, double tol, double* out,
                       int32_t* rounds_out) {
    Grid g(*d);
    Metric m(g);
    const int n = g.count();
    std::vector<std::vector<uint8_t>> fixed(batch, std::vector<uint8_t>(n, 0));
    for (int e = 0; e < batch; e++) {
        double* f = out + int64_t(e) * n;
        std::fill(f, f + n, kInf);
        for (int q = seed_off[e]; q < seed_off[e + 1]; q++) {
            int s = seed_idx[q];
            if (unsigned(s) >= unsigned(n)) continue;
            f[s] = std::min(f[s], seed_t[q]);
            fixed[e][s] = 1;
        }
    }
    const int cap = max_rounds > 0 ? max_rounds : sweep_round_cap(g);
    for (int phase = 0; phase < 2; phase++) {
        bool settled = false;
        int round = 0;
        for (round = 0; round < cap && !settled; round++) {
            bool changed = false;
            for (int e = 0; e < batch; e++)
                if (relax_round(g, m, slowness, out + int64_t(e) * n, fixed[e], phase, tol)) changed = true;
            settled = !changed;
        }
        if (rounds_out) rounds_out[phase] = round;
        if (!settled) return 0;
    }
    return 1;
}

// SphericalEikonal.Solve (SphericalEikonal.cs:102-152): fast marching, the reference's production CPU
// solver (and the timed CPU baseline). Seeds are imposed; neighbours are updated from Alive nodes only.
int32_t or_fmm(const or_grid_def* d, const double* slowness, int32_t n_seeds, const int32_t* seed_idx,
               const double* seed_t, double* out) {
    Grid g(*d);
    Metric m(g);
    int n = g.count();
    if (n_seeds == 0) return 0;
    enum : uint8_t { Far = 0, Trial = 1, Alive = 2, Seed = 3 };
    std::fill(out, out + n, kInf);
    std::vector<uint8_t> status(n, Far);
    FrontHeap heap(n, std::max(1024, n / 64));
    for (int q = 0; q < n_seeds; q++) {
        int s = seed_idx[q];
        if (unsigned(s) >= unsigned(n) || !(seed_t[q] < out[s])) continue;
        out[s] = seed_t[q];
        status[s] = Seed;
        heap.set(s, seed_t[q]);
    }
    int nx = g.nx, ny = g.ny, nz = g.nz, nxy = nx * ny;
    auto alive = [&](int node) { return status[node] == Alive; };
    // March.Axis (SphericalEikonal.cs:202-222): the term of one axis from Alive neighbours.
    auto axis = [&](int index, int pos, int nn, int stride, double h, Term* q, int& used, bool zvar, int k) {
        double minus = pos > 0 && alive(index - stride) ? out[index - stride] : kInf;
        double plus = pos + 1 < nn && alive(index + stride) ? out[index + stride] : kInf;
        double first;
        int second;
        bool minus_side = minus <= plus;
        if (minus_side) { first = minus; second = pos > 1 ? index - 2 * stride : -1; }
        else { first = plus; second = pos + 2 < nn ? index + 2 * stride : -1; }
        if (!std::isfinite(first)) return;
        double t2 = second >= 0 && alive(second) ? out[second] : kInf;
        if (!zvar) {
            if (std::isfinite(t2) && t2 <= first) q[used] = {(4 * first - t2) / 3, 2 * h / 3, first};
            else q[used] = {first, h, first};
        } else {
            double h1 = minus_side ? m.dz[k - 1] : m.dz[k];
            if (std::isfinite(t2) && t2 <= first) {
                double h2 = minus_side ? m.dz[k - 2] : m.dz[k + 1];
                double a = (2 * h1 + h2) / (h1 * (h1 + h2));
                double b = (h1 + h2) / (h1 * h2);
                double c = h1 / (h2 * (h1 + h2));
                q[used] = {(b * first - c * t2) / a, 1 / a, first};
            } else {
                q[used] = {first, h1, first};
            }
        }
        used++;
    };
    // March.SolveNode (SphericalEikonal.cs:167-200).
    auto solve_node = [&](int index, int i, int j, int k) -> double {
        double s = slowness[index];
        if (!(s > 0) || !std::isfinite(s)) return kInf;
        Term q[3];
        int used = 0;
        axis(index, i, nx, 1, m.hlon[size_t(k) * ny + j], q, used, false, k);
        axis(index, j, ny, nx, m.hlat[k], q, used, false, k);
        axis(index, k, nz, nxy, m.hr, q, used, g.variable, k);
        if (used == 0) return kInf;
        sort_terms(q, used);
        return godunov(q, used, s);
    };
    auto update = [&](int nidx, int i, int j, int k) {
        if (status[nidx] >= Alive) return;
        double t = solve_node(nidx, i, j, k);
        if (!(t < out[nidx])) return;
        out[nidx] = t;
        status[nidx] = Trial;
        heap.set(nidx, t);
    };
    int idx;
    while (heap.pop(idx)) {
        status[idx] = Alive;
        int k = idx / nxy, rest = idx - k * nxy, j = rest / nx, i = rest - j * nx;
        if (i > 0) update(idx - 1, i - 1, j, k);
        if (i + 1 < nx) update(idx + 1, i + 1, j, k);
        if (j > 0) update(idx - nx, i, j - 1, k);
        if (j + 1 < ny) update(idx + nx, i, j + 1, k);
        if (k > 0) update(idx - nxy, i, j, k - 1);
        if (k + 1 < nz) update(idx + nxy, i, j, k + 1);
    }
    return 1;
}

// Many fast-marching solves at once, one field per thread (TravelTimeTable.cs:332-354, 396-400):
// fields f uses seeds [seed_off[f], seed_off[f+1]) and slowness slowness + sl_of[f]*n.
void or_fmm_many(const or_grid_def* d, const double* slowness, const int32_t* sl_of, int32_t n_fields,
                 const int32_t* seed_off, const int32_t* seed_idx, const double* seed_t, double* out,
                 int32_t threads) {
    int n = d->nx * d->ny * d->nz;
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            int f = next.fetch_add(1);
            if (f >= n_fields) return;
            or_fmm(d, slowness + size_t(sl_of[f]) * n, seed_off[f + 1] - seed_off[f], seed_idx + seed_off[f],
                   seed_t + seed_off[f], out + size_t(f) * n);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); t++) pool.emplace_back(work);
    for (auto& t : pool) t.join();
}

// ---- tables and rays -------------------------------------------------------------------------

// TravelTimeTable.Write's float32 rounding (TravelTimeTable.cs:73).
void or_to_table(const double* t, int64_t n, float* out) {
    for (int64_t q = 0; q < n; q++) out[q] = std::isfinite(t[q]) ? float(t[q]) : std::numeric_limits<float>::infinity();
}

double or_table_time(const or_grid_def* d, const float* table, double lon, double lat, double dep) {
    Grid g(*d);
    Table tb{g, table, 0, 0, 0};
    return tb.time(lon, lat, dep);
}

void or_table_gradient(const or_grid_def* d, const float* table, double lon, double lat, double dep, double* g3) {
    Grid g(*d);
    Table tb{g, table, 0, 0, 0};
    tb.gradient(lon, lat, dep, g3[0], g3[1], g3[2]);
}

// RayTracing.Backtrack: writes up to cap points (lon, lat, depth interleaved); returns the point
// count, 0 when the reference returns null, or -needed when cap is too small.
int32_t or_backtrack(const or_grid_def* d, const float* table, double st_lon, double st_lat, double st_dep,
                     double lon, double lat, double dep, double step_km, double* pts, int32_t cap) {
    Grid g(*d);
    Table tb{g, table, st_lon, st_lat, st_dep};
    std::vector<Geo> path;
    if (!backtrack(tb, lon, lat, dep, step_km, path)) return 0;
    if (int(path.size()) > cap) return -int(path.size());
    for (size_t q = 0; q < path.size(); q++) {
        pts[3 * q] = path[q].lon; pts[3 * q + 1] = path[q].lat; pts[3 * q + 2] = path[q].depth;
    }
    return int(path.size());
}

// RayTracing.Kernel over a given polyline on the inversion grid; nodes in first-visit order.
int32_t or_kernel(const or_grid_def* inv, const double* pts, int32_t n_pts, int32_t* nodes, double* lens, int32_t cap) {
    Grid g(*inv);
    std::vector<Geo> ray(n_pts);
    for (int q = 0; q < n_pts; q++) ray[q] = {pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]};
    std::vector<int> keys;
    std::vector<double> vals;
    ray_kernel(g, ray, keys, vals);
    if (int(keys.size()) > cap) return -int(keys.size());
    for (size_t q = 0; q < keys.size(); q++) { nodes[q] = keys[q]; lens[q] = vals[q]; }
    return int(keys.size());
}

// One arrival of RayKernels.Compute (Tomography/RayKernels.cs:77-97): backtrack on the station's
// table, TCalc and the source gradient, the kernel on the inversion grid, nodes ascending, lengths
// cast to float32. Returns nnz (>= 0, an empty row is kept), -1 for an arrival the reference drops,
// or -2 - needed when cap is too small.
int32_t or_ray_row_bg(const or_grid_def* fwd, const float* table, double st_lon, double st_lat, double st_dep,
                      const or_grid_def* inv, double ev_lon, double ev_lat, double ev_dep, double step_km,
                      int32_t* nodes, float* lens, int32_t cap, double* tcalc_grad4, int32_t nbg, const double* bgd,
                      const double* bgv, double* outside);

int32_t or_ray_row(const or_grid_def* fwd, const float* table, double st_lon, double st_lat, double st_dep,
                   const or_grid_def* inv, double ev_lon, double ev_lat, double ev_dep, double step_km,
                   int32_t* nodes, float* lens, int32_t cap, double* tcalc_grad4) {
    double outside = 0;
    return or_ray_row_bg(fwd, table, st_lon, st_lat, st_dep, inv, ev_lon, ev_lat, ev_dep, step_km, nodes, lens, cap,
                         tcalc_grad4, 0, nullptr, nullptr, &outside);
}

// RayKernels.Compute's row with the extended domain's background (RayKernels.cs:63-65, 95): bgv is
// the background's Vp or Vs (the arrival's phase); *outside is RayRow.OutsideTime.
int32_t or_ray_row_bg(const or_grid_def* fwd, const float* table, double st_lon, double st_lat, double st_dep,
                      const or_grid_def* inv, double ev_lon, double ev_lat, double ev_dep, double step_km,
                      int32_t* nodes, float* lens, int32_t cap, double* tcalc_grad4, int32_t nbg, const double* bgd,
                      const double* bgv, double* outside) {
    Grid g(*fwd);
    Grid ig(*inv);
    Table tb{g, table, st_lon, st_lat, st_dep};
    std::vector<Geo> path;
    if (!backtrack(tb, ev_lon, ev_lat, ev_dep, step_km, path)) return -1;
    double tcalc = tb.time(ev_lon, ev_lat, ev_dep);
    double ge, gn, gz;
    tb.gradient(ev_lon, ev_lat, ev_dep, ge, gn, gz);
    if (!std::isfinite(tcalc)) return -1;
    std::vector<int> keys;
    std::vector<double> vals;
    ray_kernel(ig, path, keys, vals, nbg, bgd, bgv, outside);
    if (int(keys.size()) > cap) return -2 - int(keys.size());
    std::vector<int> order(keys.size());
    for (size_t q = 0; q < order.size(); q++) order[q] = int(q);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    for (size_t q = 0; q < order.size(); q++) {
        nodes[q] = keys[order[q]];
        lens[q] = float(vals[order[q]]);
    }
    tcalc_grad4[0] = tcalc; tcalc_grad4[1] = ge; tcalc_grad4[2] = gn; tcalc_grad4[3] = gz;
    return int(keys.size());
}

// Many arrivals on a thread pool (RayKernels.cs:67): arrival a traces on table tables + tab_of[a]*n
// with station st[3*a..]; writes row a's result (as or_ray_row returns it) into nnz[a] and its entries
// at [a*cap_per_row, ...).
void or_ray_rows_many(const or_grid_def* fwd, const float* tables, const int32_t* tab_of, const double* st,
                      const or_grid_def* inv, const double* ev, int32_t n_rays, double step_km, int32_t cap_per_row,
                      int32_t* nnz, int32_t* nodes, float* lens, double* tcalc_grad4, int32_t threads) {
    int64_t n = int64_t(fwd->nx) * fwd->ny * fwd->nz;
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            int a = next.fetch_add(1);
            if (a >= n_rays) return;
            nnz[a] = or_ray_row(fwd, tables + size_t(tab_of[a]) * n, st[3 * a], st[3 * a + 1], st[3 * a + 2], inv,
                                ev[3 * a], ev[3 * a + 1], ev[3 * a + 2], step_km, nodes + size_t(a) * cap_per_row,
                                lens + size_t(a) * cap_per_row, cap_per_row, tcalc_grad4 + 4 * size_t(a));
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); t++) pool.emplace_back(work);
    for (auto& t : pool) t.join();
}

// or_ray_rows_many with the background of the extended domain: tab_phase[t] picks Vp (0) or Vs (1);
// outside[a] is row a's time outside the inversion grid.
void or_ray_rows_many_bg(const or_grid_def* fwd, const float* tables, const int32_t* tab_of, const int32_t* tab_phase,
                         const double* st, const or_grid_def* inv, const double* ev, int32_t n_rays, double step_km,
                         int32_t cap_per_row, int32_t* nnz, int32_t* nodes, float* lens, double* tcalc_grad4,
                         int32_t nbg, const double* bgd, const double* bgvp, const double* bgvs, double* outside,
                         int32_t threads) {
    int64_t n = int64_t(fwd->nx) * fwd->ny * fwd->nz;
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            int a = next.fetch_add(1);
            if (a >= n_rays) return;
            const double* bgv = tab_phase[tab_of[a]] == 0 ? bgvp : bgvs;
            nnz[a] = or_ray_row_bg(fwd, tables + size_t(tab_of[a]) * n, st[3 * a], st[3 * a + 1], st[3 * a + 2], inv,
                                   ev[3 * a], ev[3 * a + 1], ev[3 * a + 2], step_km, nodes + size_t(a) * cap_per_row,
                                   lens + size_t(a) * cap_per_row, cap_per_row, tcalc_grad4 + 4 * size_t(a), nbg, bgd,
                                   bgv, outside + a);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); t++) pool.emplace_back(work);
    for (auto& t : pool) t.join();
}

// Many Relax solves on a thread pool (parity checks of batches).
void or_relax_many(const or_grid_def* d, const double* slowness, const int32_t* sl_of, int32_t n_fields,
                   const int32_t* seed_off, const int32_t* seed_idx, const double* seed_t, double tol, double* out,
                   int32_t* rounds, int32_t* settled, int32_t threads) {
    int n = d->nx * d->ny * d->nz;
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            int f = next.fetch_add(1);
            if (f >= n_fields) return;
            settled[f] = or_relax(d, slowness + size_t(sl_of[f]) * n, seed_off[f + 1] - seed_off[f],
                                  seed_idx + seed_off[f], seed_t + seed_off[f], 0, tol, out + size_t(f) * n,
                                  rounds + 2 * f);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); t++) pool.emplace_back(work);
    for (auto& t : pool) t.join();
}

}  // extern "C"

extern "C" {

// The reference's sweeping with node-level due flags (EikonalOpenCl.cs:528-532, 608-622), where a
// node wakes its 12 stencil neighbours only when it dropped by more than wake_rel of its new value
// (wake_rel = 0: every drop wakes, the reference's rule, identical to or_relax). With `causal`, a
// drop to t wakes only the neighbours holding more than t: an upwind update uses only neighbours
// smaller than its result, so a neighbour at or below t cannot be lowered by it (the engine's fast
// mode). Used to bound the effect of both rules. evals_out receives the node evaluations made.
int32_t or_relax_wake(const or_grid_def* d, const double* slowness, int32_t n_seeds, const int32_t* seed_idx,
                      const double* seed_t, double tol, double wake_rel, int32_t causal, double* out,
                      int32_t* rounds_out, int64_t* evals_out) {
    Grid g(*d);
    Metric m(g);
    int n = g.count();
    std::fill(out, out + n, kInf);
    std::vector<uint8_t> fixed(n, 0), due(n, 1);
    for (int q = 0; q < n_seeds; q++) {
        int s = seed_idx[q];
        if (unsigned(s) >= unsigned(n)) continue;
        out[s] = std::min(out[s], seed_t[q]);
        fixed[s] = 1;
    }
    int nx = g.nx, ny = g.ny, nz = g.nz, nxy = nx * ny;
    int cap = sweep_round_cap(g);
    int64_t evals = 0;
    int settled_all = 1;
    for (int phase = 0; phase < 2; phase++) {
        std::fill(due.begin(), due.end(), 1);
        int settled = 0, round = 0;
        for (round = 0; round < cap; round++) {
            bool changed = false;
            for (int dir = 0; dir < 8; dir++)
                for (int p = 0; p < nx + ny + nz - 2; p++) {
                    int i0, i1, k0, k1;
                    plane_bounds(nx, ny, nz, p, i0, i1, k0, k1);
                    for (int kp = k0; kp <= k1; kp++)
                        for (int ip = i0; ip <= i1; ip++) {
                            int jp = p - ip - kp;
                            if (jp < 0 || jp >= ny) continue;
                            int i = (dir & 1) ? nx - 1 - ip : ip;
                            int j = (dir & 2) ? ny - 1 - jp : jp;
                            int k = (dir & 4) ? nz - 1 - kp : kp;
                            int idx = g.index(i, j, k);
                            if (fixed[idx] || !due[idx]) continue;
                            due[idx] = 0;
                            evals++;
                            double cur = out[idx];
                            double cand = relax_node(m, slowness, out, idx, i, j, k, phase == 1);
                            if (!(cand < cur)) continue;
                            out[idx] = cand;
                            if (!std::isfinite(cur) || cur - cand > tol) changed = true;
                            if (std::isfinite(cur) && cur - cand <= wake_rel * cand) continue;
                            auto wake = [&](int nb) {
                                if (!causal || cand < out[nb]) due[nb] = 1;
                            };
                            for (int s = 1; s <= 2; s++) {
                                if (i >= s) wake(idx - s);
                                if (i + s < nx) wake(idx + s);
                                if (j >= s) wake(idx - s * nx);
                                if (j + s < ny) wake(idx + s * nx);
                                if (k >= s) wake(idx - s * nxy);
                                if (k + s < nz) wake(idx + s * nxy);
                            }
                        }
                }
            if (!changed) { settled = 1; round++; break; }
        }
        if (rounds_out) rounds_out[phase] = round;
        if (!settled) settled_all = 0;
    }
    if (evals_out) *evals_out = evals;
    return settled_all;
}

}  // extern "C"

extern "C" {

// ---- LSQR (Numerics/Lsqr.cs:33-152): damped LSQR of Paige & Saunders on a CSR matrix --------------
// Sequential sums throughout; the transpose product is built the reference's way (CsrMatrix.Transpose,
// SparseMatrix.cs:79-96: a stable counting sort by column, rows ascending within a column).
// Stop codes: 0 empty system, 1 zero right-hand side, 2 Aᵀb = 0, 3 iteration budget, 4 btol,
// 5 atol, 6 conlim, 7 residual at machine precision, 8 normal equations at machine precision,
// 9 condition number at machine precision, 10 bidiagonalisation terminated.
// info[4]: iterations, ‖b‖, ‖r‖, condition estimate.

static double lsqr_dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0;
    for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
    return s;
}

// SimdVector.Norm (Numerics/SimdVector.cs:33-45): scaled when the entries are extreme.
static double lsqr_norm(const std::vector<double>& a) {
    double mx = 0;
    for (double x : a) mx = std::max(mx, std::fabs(x));
    if (mx == 0 || !std::isfinite(mx)) return mx;
    if (mx > 1e150 || mx < 1e-150) {
        double s = 0, inv = 1.0 / mx;
        for (double x : a) { double y = x * inv; s += y * y; }
        return mx * std::sqrt(s);
    }
    return std::sqrt(lsqr_dot(a, a));
}

static void csr_mul(int32_t rows, const int32_t* rs, const int32_t* ci, const double* va, const std::vector<double>& x,
                    std::vector<double>& y) {
    for (int32_t i = 0; i < rows; i++) {
        double s = 0;
        for (int32_t k = rs[i]; k < rs[i + 1]; k++) s += va[k] * x[ci[k]];
        y[i] = s;
    }
}

// The products or_lsqr forms (CsrMatrix.MultiplyInto, SparseMatrix.cs:55-72: one sequential sum per
// row), exported for the comparison with the reference's own spmv kernel (LsqrOpenCl.cs:45-53).
void or_csr_mul(int32_t rows, const int32_t* rs, const int32_t* ci, const double* va, const double* x, double* y) {
    for (int32_t i = 0; i < rows; i++) {
        double s = 0;
        for (int32_t k = rs[i]; k < rs[i + 1]; k++) s += va[k] * x[ci[k]];
        y[i] = s;
    }
}

// CsrMatrix.Transpose (SparseMatrix.cs:79-96) as or_lsqr builds it: a stable counting sort by column.
void or_csr_transpose(int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col, const double* val,
                      int32_t* trs, int32_t* tci, double* tva) {
    const int64_t nnz = row_ptr[m];
    for (int32_t c = 0; c <= n; c++) trs[c] = 0;
    for (int64_t k = 0; k < nnz; k++) trs[col[k] + 1]++;
    for (int32_t c = 0; c < n; c++) trs[c + 1] += trs[c];
    std::vector<int32_t> next(trs, trs + n);
    for (int32_t i = 0; i < m; i++)
        for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) {
            int32_t p = next[col[k]]++;
            tci[p] = i;
            tva[p] = val[k];
        }
}

int32_t or_lsqr(int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col, const double* val, const double* b,
                double damp, int32_t max_iterations, double atol, double btol, double conlim, double* x_out,
                double* info) {
    std::vector<double> x(n, 0.0);
    auto done = [&](int code, int it, double bn, double rn, double ac) {
        for (int32_t j = 0; j < n; j++) x_out[j] = x[j];
        info[0] = it; info[1] = bn; info[2] = rn; info[3] = ac;
        return code;
    };
    if (m == 0 || n == 0) return done(0, 0, 0, 0, 0);
    // Transpose (CsrMatrix.Transpose).
    const int64_t nnz = row_ptr[m];
    std::vector<int32_t> trs(n + 1, 0), tci(nnz);
    std::vector<double> tva(nnz);
    for (int64_t k = 0; k < nnz; k++) trs[col[k] + 1]++;
    for (int32_t c = 0; c < n; c++) trs[c + 1] += trs[c];
    std::vector<int32_t> next(trs.begin(), trs.end() - 1);
    for (int32_t i = 0; i < m; i++)
        for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) {
            int32_t p = next[col[k]]++;
            tci[p] = i;
            tva[p] = val[k];
        }
    std::vector<double> u(b, b + m), v(n), w(n), tm(m), tn(n);
    double beta = lsqr_norm(u);
    if (beta == 0) return done(1, 0, 0, 0, 0);
    const double bnorm = beta;
    for (auto& e : u) e *= 1.0 / beta;
    csr_mul(n, trs.data(), tci.data(), tva.data(), u, v);
    double alpha = lsqr_norm(v);
    if (alpha == 0) return done(2, 0, bnorm, bnorm, 0);
    for (auto& e : v) e *= 1.0 / alpha;
    w = v;
    double rhobar = alpha, phibar = beta;
    double ddnorm = 0, xxnorm = 0, z = 0, cs2 = -1, sn2 = 0, anorm2 = 0, damped2 = 0, rnorm = beta, acond = 0;
    const double ctol = conlim > 0 ? 1.0 / conlim : 0.0;
    int stop = 3, it = 0;
    for (int k = 0; k < max_iterations; k++) {
        it = k + 1;
        csr_mul(m, row_ptr, col, val, v, tm);
        for (int32_t i = 0; i < m; i++) u[i] = tm[i] - alpha * u[i];
        beta = lsqr_norm(u);
        if (beta > 0) {
            for (auto& e : u) e *= 1.0 / beta;
            anorm2 += alpha * alpha + beta * beta + damp * damp;
            csr_mul(n, trs.data(), tci.data(), tva.data(), u, tn);
            for (int32_t j = 0; j < n; j++) v[j] = tn[j] - beta * v[j];
            alpha = lsqr_norm(v);
            if (alpha > 0) for (auto& e : v) e *= 1.0 / alpha;
        }
        double rhobar1 = std::sqrt(rhobar * rhobar + damp * damp);
        double cs1 = rhobar / rhobar1, sn1 = damp / rhobar1;
        double psi = sn1 * phibar;
        phibar = cs1 * phibar;
        double rho = std::sqrt(rhobar1 * rhobar1 + beta * beta);
        double cs = rhobar1 / rho, sn = beta / rho;
        double theta = sn * alpha;
        rhobar = -cs * alpha;
        double phi = cs * phibar;
        phibar = sn * phibar;
        double tau = sn * phi;
        ddnorm += lsqr_dot(w, w) / (rho * rho);
        double t1c = phi / rho, t2c = -theta / rho;
        for (int32_t j = 0; j < n; j++) x[j] += t1c * w[j];
        for (int32_t j = 0; j < n; j++) w[j] = v[j] + t2c * w[j];
        double delta = sn2 * rho, gambar = -cs2 * rho, rhs = phi - delta * z;
        double gamma = std::sqrt(gambar * gambar + theta * theta);
        cs2 = gambar / gamma;
        sn2 = theta / gamma;
        z = rhs / gamma;
        xxnorm += z * z;
        damped2 += psi * psi;
        double anorm = std::sqrt(anorm2);
        acond = anorm * std::sqrt(ddnorm);
        double arnorm = alpha * std::fabs(tau);
        rnorm = std::sqrt(phibar * phibar + damped2);
        double xnorm = std::sqrt(xxnorm);
        double test1 = rnorm / bnorm;
        double test2 = arnorm / std::max(1e-300, anorm * rnorm);
        double test3 = 1.0 / std::max(1e-300, acond);
        double t1 = test1 / (1 + anorm * xnorm / bnorm);
        double rtol = btol + atol * anorm * xnorm / bnorm;
        if (test1 <= rtol) { stop = 4; break; }
        if (test2 <= atol) { stop = 5; break; }
        if (ctol > 0 && test3 <= ctol) { stop = 6; break; }
        if (1 + t1 <= 1) { stop = 7; break; }
        if (1 + test2 <= 1) { stop = 8; break; }
        if (1 + test3 <= 1) { stop = 9; break; }
        if (beta == 0 || alpha == 0) { stop = 10; break; }
    }
    return done(stop, it, bnorm, rnorm, acond);
}

}  // extern "C"

// ---- Event location (Location/EventLocator.cs:59-342, Relocation.Absolute's per-event loop,
// Location/Relocation.cs:48-97) -----------------------------------------------------------------
// Settings and result follow LocatorSettings (EventLocator.cs:10-36) and LocationResult + Hypocentre
// (EventLocator.cs:38, Model/Catalogue.cs:92-114). An event's observations are its usable picks with
// a table (EventLocator.cs:64-73): the table, the pick time in s after the event's reference time,
// the weight and the station correction. t0 is the origin time in s after the reference time.

namespace {

struct LocSettings {
    int32_t global_search, coarse_candidates, max_geiger_iterations, min_phases;
    double damping, outlier_mads, outlier_floor;
    int32_t fix_depth, reserved;
};

struct LocResult {
    double t0, lon, lat, depth_km, rms, err_h_km, err_minor_km, err_azimuth_deg, err_depth_km, err_time_s, gap_deg;
    int32_t used, rejected, iterations, status;
};

struct LocObs {
    const float* table;
    double obs, weight, corr, st_lon, st_lat;
};

// Math.Max / Math.Min / Math.Clamp of .NET: NaN propagates, +0 preferred over -0 by Max.
inline double net_max(double a, double b) {
    if (std::isnan(a) || std::isnan(b)) return std::nan("");
    if (a == b) return std::signbit(a) ? b : a;
    return a > b ? a : b;
}
inline double net_clamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

// DateTime.AddSeconds then (OriginTime - reference).TotalSeconds: t0 truncated to 100 ns ticks
// (integral and fractional parts converted separately), then ticks / 1e7.
inline double tick_seconds(double t0) {
    double ip = std::trunc(t0);
    double fp = t0 - ip;
    int64_t ticks = int64_t(ip) * 10000000LL + int64_t(fp * 10000000.0);
    return double(ticks) / 10000000.0;
}

// EventLocator.WeightedMedian (EventLocator.cs:297-309): NaN dropped, stable sort by value, the first
// value whose running weight reaches half the total.
double weighted_median(const std::vector<double>& v, const std::vector<double>& w) {
    std::vector<std::pair<double, double>> p;
    for (size_t i = 0; i < v.size(); i++)
        if (!std::isnan(v[i])) p.push_back({v[i], w[i]});
    std::stable_sort(p.begin(), p.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    if (p.empty()) return 0;
    double sum = 0;
    for (auto& e : p) sum += e.second;
    double half = sum / 2, acc = 0;
    for (auto& e : p) {
        acc += e.second;
        if (acc >= half) return e.first;
    }
    return p.back().first;
}

// EventLocator.Median (EventLocator.cs:311-317).
double plain_median(const std::vector<double>& v) {
    std::vector<double> s;
    for (double x : v)
        if (!std::isnan(x)) s.push_back(x);
    if (s.empty()) return 0;
    std::stable_sort(s.begin(), s.end(), [](double a, double b) { return a < b; });
    size_t n = s.size();
    return n % 2 == 1 ? s[n / 2] : 0.5 * (s[n / 2 - 1] + s[n / 2]);
}

// EventLocator.Gap (EventLocator.cs:320-327).
double azimuth_gap(std::vector<double> az) {
    std::vector<double> a;
    for (double x : az)
        if (std::find(a.begin(), a.end(), x) == a.end()) a.push_back(x);
    std::sort(a.begin(), a.end());
    if (a.size() < 2) return 360;
    double gap = 360 - a.back() + a[0];
    for (size_t i = 1; i < a.size(); i++) gap = std::max(gap, a[i] - a[i - 1]);
    return gap;
}

// GeoMath.Azimuth (Geo/GeoMath.cs:98-107).
double azimuth_deg(double lon1, double lat1, double lon2, double lat2) {
    double p1 = lat1 * kDeg2Rad, p2 = lat2 * kDeg2Rad, dl = (lon2 - lon1) * kDeg2Rad;
    double y = std::sin(dl) * std::cos(p2);
    double x = std::cos(p1) * std::sin(p2) - std::sin(p1) * std::cos(p2) * std::cos(dl);
    double az = std::atan2(y, x) * kRad2Deg;
    return std::fmod(az + 360, 360);
}

// GeoMath.NormalizeLon and GeoMath.Destination (Geo/GeoMath.cs:123-138).
double normalize_lon(double lon) {
    lon = std::fmod(lon + 180, 360);
    if (lon < 0) lon += 360;
    return lon - 180;
}
void destination(double lon, double lat, double az_deg, double dist_km, double& lon2, double& lat2) {
    double d = dist_km / kEarthRadiusKm;
    double p1 = lat * kDeg2Rad, l1 = lon * kDeg2Rad, az = az_deg * kDeg2Rad;
    double p2 = std::asin(std::sin(p1) * std::cos(d) + std::cos(p1) * std::sin(d) * std::cos(az));
    double l2 = l1 + std::atan2(std::sin(az) * std::sin(d) * std::cos(p1), std::cos(d) - std::sin(p1) * std::sin(p2));
    lon2 = normalize_lon(l2 * kRad2Deg);
    lat2 = p2 * kRad2Deg;
}

// EventLocator.Solve (EventLocator.cs:259-282): Gauss-Jordan with partial pivoting; false for null.
bool solve_small(const double a[4][4], const double* b, int n, double* x) {
    double m[4][5];
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) m[i][j] = a[i][j];
        m[i][n] = b[i];
    }
    for (int c = 0; c < n; c++) {
        int p = c;
        for (int r = c + 1; r < n; r++)
            if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
        if (std::fabs(m[p][c]) < 1e-30) return false;
        if (p != c)
            for (int j = 0; j <= n; j++) std::swap(m[c][j], m[p][j]);
        for (int r = 0; r < n; r++) {
            if (r == c) continue;
            double f = m[r][c] / m[c][c];
            for (int j = c; j <= n; j++) m[r][j] -= f * m[c][j];
        }
    }
    for (int i = 0; i < n; i++) x[i] = m[i][n] / m[i][i];
    return true;
}

}  // namespace

namespace {

struct Locator {
    const Grid& g;
    const LocSettings& s;

    // GridSearch's Misfit (EventLocator.cs:111-124): weighted median origin time, weighted L1 misfit.
    double node_misfit(const std::vector<LocObs>& obs, int idx, double& t0) const {
        std::vector<double> r(obs.size()), w(obs.size());
        for (size_t q = 0; q < obs.size(); q++) {
            float t = obs[q].table[idx];
            r[q] = std::isfinite(t) ? obs[q].obs - double(t) - obs[q].corr : std::nan("");
            w[q] = obs[q].weight;
        }
        t0 = weighted_median(r, w);
        double m = 0;
        for (size_t q = 0; q < obs.size(); q++) m += std::isnan(r[q]) ? 10 * w[q] : w[q] * std::fabs(r[q] - t0);
        return m;
    }

    // Search (EventLocator.cs:143-163).
    int search(const std::vector<LocObs>& obs, double start_dep, double start_lon, double start_lat, int i0, int i1,
               int j0, int j1, int k0, int k1, int stride) const {
        i0 = std::max(0, i0); j0 = std::max(0, j0); k0 = std::max(0, k0);
        i1 = std::min(g.nx - 1, i1); j1 = std::min(g.ny - 1, j1); k1 = std::min(g.nz - 1, k1);
        int best = -1;
        double best_m = kInf;
        if (s.fix_depth) {
            double fx, fy, fz;
            g.fractional(start_lon, start_lat, start_dep, fx, fy, fz);
            k0 = k1 = std::clamp(int(std::nearbyint(fz)), 0, g.nz - 1);
        }
        // A box wholly outside the grid (a local search from a start far outside it): the reference
        // would read past its table and Relocation.Absolute reports the exception; here -1.
        if (i0 > i1 || j0 > j1 || k0 > k1) return -1;
        for (int kk = k0; kk <= k1; kk += stride)
            for (int jj = j0; jj <= j1; jj += stride)
                for (int ii = i0; ii <= i1; ii += stride) {
                    int idx = g.index(ii, jj, kk);
                    double t0;
                    double m = node_misfit(obs, idx, t0);
                    if (m < best_m) { best_m = m; best = idx; }
                }
        return best < 0 ? g.index(i0, j0, k0) : best;
    }

    // GridSearch (EventLocator.cs:107-141).
    bool grid_search(const std::vector<LocObs>& obs, double slon, double slat, double sdep, double& lon, double& lat,
                     double& dep, double& t0) const {
        int best;
        if (s.global_search) {
            int stride = std::max(1, int(std::ceil(std::cbrt(double(g.count()) / s.coarse_candidates))));
            best = search(obs, sdep, slon, slat, 0, g.nx - 1, 0, g.ny - 1, 0, g.nz - 1, stride);
            int bk = best / (g.nx * g.ny), bj = (best / g.nx) % g.ny, bi = best % g.nx;
            best = search(obs, sdep, slon, slat, bi - 2 * stride, bi + 2 * stride, bj - 2 * stride, bj + 2 * stride,
                          bk - 2 * stride, bk + 2 * stride, 1);
        } else {
            double fx, fy, fz;
            g.fractional(slon, slat, sdep, fx, fy, fz);
            int ci = int(std::nearbyint(fx)), cj = int(std::nearbyint(fy)), ck = int(std::nearbyint(fz));
            best = search(obs, sdep, slon, slat, ci - 6, ci + 6, cj - 6, cj + 6, ck - 6, ck + 6, 1);
            if (best < 0) return false;
        }
        int k = best / (g.nx * g.ny), j = (best / g.nx) % g.ny, i = best % g.nx;
        node_misfit(obs, best, t0);
        lon = g.lon[i];
        lat = g.lat[j];
        dep = s.fix_depth ? sdep : g.dep[k];
        return true;
    }

    // Geiger's Misfit (EventLocator.cs:173-198).
    double geiger_misfit(const std::vector<LocObs>& obs, int npar, double x, double y, double z, double t, bool normal,
                         double ata[4][4], double* atb) const {
        if (normal) {
            std::memset(ata, 0, sizeof(double) * 16);
            std::memset(atb, 0, sizeof(double) * 4);
        }
        double sum = 0;
        int rows = 0;
        for (const LocObs& o : obs) {
            Table tb{g, o.table, 0, 0, 0};
            double tt = tb.time(x, y, z);
            if (!std::isfinite(tt)) continue;
            double res = o.obs - t - tt - o.corr;
            double w = o.weight * o.weight;
            sum += w * res * res;
            rows++;
            if (!normal) continue;
            double ge, gn, gz;
            tb.gradient(x, y, z, ge, gn, gz);
            double row[4] = {1, ge, gn, gz};
            for (int a = 0; a < npar; a++) {
                atb[a] += w * row[a] * res;
                for (int b = 0; b < npar; b++) ata[a][b] += w * row[a] * row[b];
            }
        }
        return rows >= npar ? sum : kInf;
    }

    // Geiger (EventLocator.cs:166-256).
    int geiger(const std::vector<LocObs>& obs, double& lon, double& lat, double& dep, double& t0, LocResult& out) const {
        const int npar = s.fix_depth ? 3 : 4;
        double ata[4][4], atb[4];
        double lambda = net_max(1e-6, s.damping);
        double chi2 = geiger_misfit(obs, npar, lon, lat, dep, t0, true, ata, atb);
        int it = 0;
        for (; it < s.max_geiger_iterations && std::isfinite(chi2); it++) {
            bool accepted = false, have_step = false;
            double step[4] = {0, 0, 0, 0};
            while (lambda < 1e8) {
                double lhs[4][4];
                std::memcpy(lhs, ata, sizeof lhs);
                for (int a = 0; a < npar; a++) lhs[a][a] *= 1 + lambda;
                have_step = solve_small(lhs, atb, npar, step);
                if (!have_step) break;
                double nlon, nlat;
                destination(lon, lat, std::atan2(step[1], step[2]) * kRad2Deg,
                            std::sqrt(step[1] * step[1] + step[2] * step[2]), nlon, nlat);
                double tlon = net_clamp(unwrap_lon(nlon, g.centre_lon), g.lon[0], g.lon[g.nx - 1]);
                double tlat = net_clamp(nlat, g.lat[0], g.lat[g.ny - 1]);
                double tdep = s.fix_depth ? dep : net_clamp(dep + step[3], g.dep[0], g.dep[g.nz - 1]);
                double tt0 = t0 + step[0];
                double trial = geiger_misfit(obs, npar, tlon, tlat, tdep, tt0, false, ata, atb);
                if (trial <= chi2) {
                    lon = tlon; lat = tlat; dep = tdep; t0 = tt0;
                    chi2 = geiger_misfit(obs, npar, lon, lat, dep, t0, true, ata, atb);
                    lambda = net_max(1e-6, lambda / 10);
                    accepted = true;
                    break;
                }
                lambda *= 10;
            }
            if (!accepted || !have_step) break;
            double moved = std::sqrt(step[1] * step[1] + step[2] * step[2] + (npar > 3 ? step[3] * step[3] : 0));
            if (moved < 0.005 && std::fabs(step[0]) < 0.001) { it++; break; }
        }
        geiger_misfit(obs, npar, lon, lat, dep, t0, true, ata, atb);
        double ss = 0;
        for (const LocObs& o : obs) {
            Table tb{g, o.table, 0, 0, 0};
            double r = o.obs - t0 - tb.time(lon, lat, dep) - o.corr;
            ss += r * r;
        }
        out.t0 = t0; out.lon = lon; out.lat = lat; out.depth_km = dep;
        out.rms = std::sqrt(ss / double(obs.size()));
        out.err_h_km = out.err_minor_km = out.err_azimuth_deg = out.err_depth_km = out.err_time_s = std::nan("");
        // Invert (EventLocator.cs:284-295): column by column.
        double cov[4][4];
        bool ok = true;
        for (int c = 0; c < npar && ok; c++) {
            double e[4] = {0, 0, 0, 0}, col[4];
            e[c] = 1;
            ok = solve_small(ata, e, npar, col);
            for (int r = 0; ok && r < npar; r++) cov[r][c] = col[r];
        }
        if (ok) {
            double dof = std::max(1, int(obs.size()) - npar);
            double scale = net_max(1, chi2 / dof);
            double cee = cov[1][1] * scale, cnn = cov[2][2] * scale, cen = cov[1][2] * scale;
            double tr = 0.5 * (cee + cnn);
            double det = cee * cnn - cen * cen;
            double root = std::sqrt(net_max(0, tr * tr - det));
            out.err_h_km = std::sqrt(net_max(0, tr + root));
            out.err_minor_km = std::sqrt(net_max(0, tr - root));
            double theta = 0.5 * std::atan2(2 * cen, cee - cnn) * kRad2Deg;
            out.err_azimuth_deg = std::fmod(std::fmod(90 - theta, 180) + 180, 180);
            out.err_depth_km = npar > 3 ? std::sqrt(net_max(0, cov[3][3] * scale)) : 0;
            out.err_time_s = std::sqrt(net_max(0, cov[0][0] * scale));
        }
        return it;
    }

    // Locate (EventLocator.cs:59-104). residual[q] for every observation (NaN when not located).
    LocResult locate(const std::vector<LocObs>& all, double slon, double slat, double sdep, double* residual) const {
        LocResult out{};
        out.t0 = 0; out.lon = slon; out.lat = slat; out.depth_km = sdep;
        out.rms = out.err_h_km = out.err_minor_km = out.err_azimuth_deg = out.err_depth_km = out.err_time_s =
            out.gap_deg = std::nan("");
        for (size_t q = 0; q < all.size(); q++) residual[q] = std::nan("");
        if (int(all.size()) < s.min_phases) {
            out.used = int(all.size());
            out.status = 1;
            return out;
        }
        std::vector<LocObs> used = all;
        int rejected = 0, iterations = 0;
        LocResult best{};
        for (int round = 0; round < 3; round++) {
            double lon, lat, dep, t0;
            if (!grid_search(used, slon, slat, sdep, lon, lat, dep, t0)) {
                out.status = 2;  // Relocation.Absolute's exception result: start kept, nothing used
                return out;
            }
            iterations = geiger(used, lon, lat, dep, t0, best);
            const double tq = tick_seconds(best.t0);
            std::vector<double> res(used.size());
            for (size_t q = 0; q < used.size(); q++) {
                Table tb{g, used[q].table, 0, 0, 0};
                res[q] = used[q].obs - tq - tb.time(best.lon, best.lat, best.depth_km) - used[q].corr;
            }
            double med = plain_median(res);
            std::vector<double> dev(res.size());
            for (size_t q = 0; q < res.size(); q++) dev[q] = std::fabs(res[q] - med);
            double mad = 1.4826 * plain_median(dev);
            double limit = net_max(s.outlier_floor, s.outlier_mads * mad);
            std::vector<LocObs> keep;
            for (size_t q = 0; q < used.size(); q++)
                if (std::fabs(res[q] - med) <= limit) keep.push_back(used[q]);
            if (keep.size() == used.size() || int(keep.size()) < s.min_phases) break;
            rejected += int(used.size() - keep.size());
            used = keep;
        }
        const double tq = tick_seconds(best.t0);
        for (size_t q = 0; q < all.size(); q++) {
            Table tb{g, all[q].table, 0, 0, 0};
            residual[q] = all[q].obs - tq - tb.time(best.lon, best.lat, best.depth_km) - all[q].corr;
        }
        std::vector<double> az;
        for (const LocObs& o : used) az.push_back(azimuth_deg(best.lon, best.lat, o.st_lon, o.st_lat));
        best.gap_deg = azimuth_gap(az);
        best.used = int(used.size());
        best.rejected = rejected;
        best.iterations = iterations;
        best.status = 0;
        return best;
    }
};

}  // namespace

extern "C" {

// Relocation.Absolute's loop (Location/Relocation.cs:76-91): every event located on its own,
// events spread over n_threads host threads. tables: n_tables float32 fields on g; table_station:
// lon, lat of each table's station; start: lon, lat, depth per event; out: 16 x 8 bytes per event
// (LocResult); residual: one per observation.
void or_locate_many(const or_grid_def* d, const float* tables, int32_t n_tables, const double* table_station,
                    const void* settings, int32_t n_events, const double* start, const int32_t* obs_offsets,
                    const int32_t* obs_table, const double* obs_seconds, const double* obs_weight,
                    const double* obs_corr, int32_t n_threads, void* out, double* residual) {
    Grid g(*d);
    const LocSettings& s = *static_cast<const LocSettings*>(settings);
    LocResult* res = static_cast<LocResult*>(out);
    const int64_t n = g.count();
    Locator loc{g, s};
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int e = next++; e < n_events; e = next++) {
            std::vector<LocObs> obs;
            for (int q = obs_offsets[e]; q < obs_offsets[e + 1]; q++) {
                int t = obs_table[q];
                obs.push_back({tables + int64_t(t) * n, obs_seconds[q], obs_weight[q], obs_corr[q],
                               table_station[2 * t], table_station[2 * t + 1]});
            }
            res[e] = loc.locate(obs, start[3 * e], start[3 * e + 1], start[3 * e + 2], residual + obs_offsets[e]);
        }
    };
    (void)n_tables;
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(1, n_threads); t++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
}

// WeightedMedian, Median and Gap on their own (known-answer tests).
double or_weighted_median(int32_t n, const double* v, const double* w) {
    return weighted_median(std::vector<double>(v, v + n), std::vector<double>(w, w + n));
}
double or_median(int32_t n, const double* v) { return plain_median(std::vector<double>(v, v + n)); }
double or_gap(int32_t n, const double* az) { return azimuth_gap(std::vector<double>(az, az + n)); }
double or_tick_seconds(double t0) { return tick_seconds(t0); }

}  // extern "C"

// ---- Forward domain and model (Forward/ForwardDomain.cs:51-107, Forward/TravelTimeTable.cs:217-241,
// Model/VelocityModel1D.cs:31-45) ----------------------------------------------------------------

namespace {

// VelocityModel1D.Evaluate.
double evaluate_1d(const double* depth, const double* v, int n, double d) {
    if (d <= depth[0]) return v[0];
    for (int i = 1; i < n; i++) {
        double a = depth[i - 1], b = depth[i];
        if (d > b) continue;
        if (b - a <= 1e-12) continue;
        double t = (d - a) / (b - a);
        return v[i - 1] + t * (v[i] - v[i - 1]);
    }
    return v[n - 1];
}

// SphericalGrid.Contains (Geo/SphericalGrid.cs:186-192).
bool grid_contains(const Grid& g, double lon, double lat, double dep, double tol) {
    double fx, fy, fz;
    g.fractional(lon, lat, dep, fx, fy, fz);
    return fx >= -tol && fx <= g.nx - 1 + tol && fy >= -tol && fy <= g.ny - 1 + tol && fz >= -tol && fz <= g.nz - 1 + tol;
}

}  // namespace

extern "C" {

// ForwardModel.FromInversionGrid: velocities 1/inv_slowness resampled to the forward nodes
// (ResampleFrom = Interpolate at LonDeg[i], LatDeg[j], DepthKm[k]); with a background (nbg > 0),
// nodes outside the inversion grid (tolerance 1e-6) take its Vp (phase 0) or Vs (phase 1); then 1/v.
void or_resample(const or_grid_def* fwd, const or_grid_def* inv, const double* inv_slowness, int32_t n_phases,
                 int32_t nbg, const double* bg_depth, const double* bg_vp, const double* bg_vs, double* out) {
    Grid f(*fwd), g(*inv);
    const int64_t fn = f.count(), in = g.count();
    for (int p = 0; p < n_phases; p++) {
        std::vector<double> v(in);
        for (int64_t q = 0; q < in; q++) v[q] = 1 / inv_slowness[p * in + q];
        for (int k = 0; k < f.nz; k++)
            for (int j = 0; j < f.ny; j++)
                for (int i = 0; i < f.nx; i++) {
                    double x = g.interpolate(v.data(), f.lon[i], f.lat[j], f.dep[k]);
                    if (nbg > 0 && !grid_contains(g, f.lon[i], f.lat[j], f.dep[k], 1e-6))
                        x = evaluate_1d(bg_depth, p == 0 ? bg_vp : bg_vs, nbg, f.dep[k]);
                    out[p * fn + f.index(i, j, k)] = 1 / x;
                }
    }
}

// ForwardDomain.Covering; returns 0, or 1 when the points span the globe. Refined is
// GridDefinition.Refined (Geo/SphericalGrid.cs:51-56).
int32_t or_covering(const or_grid_def* inv, int32_t refinement, int32_t n_points, const double* points,
                    int64_t max_nodes, or_grid_def* out, int32_t* extended, double* coarsening) {
    const int fct = std::max(1, refinement);
    or_grid_def fine = *inv;
    if (fct > 1) {
        fine.nx = (inv->nx - 1) * fct + 1;
        fine.ny = (inv->ny - 1) * fct + 1;
        fine.nz = (inv->nz - 1) * fct + 1;
    }
    const double fdlon = (fine.max_lon - fine.min_lon) / std::max(1, fine.nx - 1);
    const double fdlat = (fine.max_lat - fine.min_lat) / std::max(1, fine.ny - 1);
    const double fddep = (fine.max_depth_km - fine.min_depth_km) / std::max(1, fine.nz - 1);
    const double centre = 0.5 * (inv->min_lon + inv->max_lon);
    double min_lon = inv->min_lon, max_lon = inv->max_lon, min_lat = inv->min_lat, max_lat = inv->max_lat;
    double top = inv->min_depth_km, bottom = inv->max_depth_km;
    int outside = 0;
    for (int q = 0; q < n_points; q++) {
        double lon = unwrap_lon(points[3 * q], centre), lat = points[3 * q + 1], dep = points[3 * q + 2];
        bool inside = lon >= inv->min_lon && lon <= inv->max_lon && lat >= inv->min_lat && lat <= inv->max_lat &&
                      dep >= inv->min_depth_km && dep <= inv->max_depth_km;
        if (inside) continue;
        outside++;
        min_lon = std::min(min_lon, lon); max_lon = std::max(max_lon, lon);
        min_lat = std::min(min_lat, lat); max_lat = std::max(max_lat, lat);
        bottom = std::max(bottom, dep);
    }
    *extended = outside > 0;
    *coarsening = 1.0;
    if (outside == 0) {
        *out = fine;
        out->depth_km = nullptr;
        return 0;
    }
    min_lon -= 2 * fdlon; max_lon += 2 * fdlon;
    min_lat = std::max(-89.0, min_lat - 2 * fdlat); max_lat = std::min(89.0, max_lat + 2 * fdlat);
    if (bottom > inv->max_depth_km) bottom += 2 * fddep;
    if (max_lon - min_lon >= 359) return 1;
    double dlon = fdlon, dlat = fdlat, ddep = fddep;
    auto count = [&](double f) {
        return int64_t(std::ceil((max_lon - min_lon) / (dlon * f)) + 1) * int64_t(std::ceil((max_lat - min_lat) / (dlat * f)) + 1) *
               int64_t(std::ceil((bottom - top) / (ddep * f)) + 1);
    };
    double factor = 1.0;
    while (count(factor) > max_nodes) factor *= 1.25;
    dlon *= factor; dlat *= factor; ddep *= factor;
    int west = int(std::ceil((inv->min_lon - min_lon) / dlon)), east = int(std::ceil((max_lon - inv->max_lon) / dlon));
    int south = int(std::ceil((inv->min_lat - min_lat) / dlat)), north = int(std::ceil((max_lat - inv->max_lat) / dlat));
    int down = int(std::ceil((bottom - inv->max_depth_km) / ddep));
    int nx = int(std::nearbyint((inv->max_lon - inv->min_lon) / dlon));
    int ny = int(std::nearbyint((inv->max_lat - inv->min_lat) / dlat));
    int nz = int(std::nearbyint((inv->max_depth_km - inv->min_depth_km) / ddep));
    or_grid_def d{};
    d.min_lon = inv->min_lon - west * dlon;
    d.max_lon = inv->min_lon - west * dlon + (west + nx + east) * dlon;
    d.min_lat = inv->min_lat - south * dlat;
    d.max_lat = inv->min_lat - south * dlat + (south + ny + north) * dlat;
    d.min_depth_km = inv->min_depth_km;
    d.max_depth_km = inv->min_depth_km + (nz + down) * ddep;
    d.nx = west + nx + east + 1; d.ny = south + ny + north + 1; d.nz = nz + down + 1;
    d.depth_km = nullptr;
    *out = d;
    *coarsening = factor;
    return 0;
}

double or_background(const double* depth, const double* v, int32_t n, double d) { return evaluate_1d(depth, v, n, d); }

}  // extern "C"
