// The self-test gate's host solver (EikonalOpenCl.SelfTest compares the device with
// SphericalEikonal.Relax on the host, Forward/EikonalOpenCl.cs:346-374). Used by ts_cuda_selftest
// only; no solve ever returns its result. Compiled with -ffp-contract=off.
#include <algorithm>
#include <cmath>

#include "host_geo.h"

namespace ts {
namespace host {

namespace {

struct Term {
    double t, h, n;
};

// RelaxNode (Forward/SphericalEikonal.cs:349-396) on a uniform grid.
double relax_node(const Grid& g, const Metric& m, const double* slow, const double* f, int idx, int i, int j, int k,
                  bool second) {
    double s = slow[idx];
    if (!(s > 0)) return kInf;
    const int nx = g.nx, ny = g.ny, nz = g.nz, nxy = nx * ny;
    Term q[3];
    int used = 0;
    auto axis = [&](int pos, int n, int stride, double h) {
        double minus = pos > 0 ? f[idx - stride] : kInf;
        double plus = pos + 1 < n ? f[idx + stride] : kInf;
        double first, t2;
        if (minus <= plus) { first = minus; t2 = pos > 1 ? f[idx - 2 * stride] : kInf; }
        else { first = plus; t2 = pos + 2 < n ? f[idx + 2 * stride] : kInf; }
        if (!std::isfinite(first)) return;
        if (!second) t2 = kInf;
        if (std::isfinite(t2) && t2 <= first) q[used] = {(4 * first - t2) / 3, 2 * h / 3, first};
        else q[used] = {first, h, first};
        used++;
    };
    axis(i, nx, 1, m.hlon[size_t(k) * ny + j]);
    axis(j, ny, nx, m.hlat[k]);
    axis(k, nz, nxy, m.hr);
    if (used == 0) return kInf;
    for (int a = 1; a < used; a++) {
        Term x = q[a];
        int b = a - 1;
        while (b >= 0 && q[b].t > x.t) { q[b + 1] = q[b]; b--; }
        q[b + 1] = x;
    }
    for (int terms = used; terms >= 1; terms--) {
        double sw = 0, swt = 0, swt2 = 0;
        for (int r = 0; r < terms; r++) {
            double w = 1.0 / (q[r].h * q[r].h);
            sw += w; swt += w * q[r].t; swt2 += w * q[r].t * q[r].t;
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

}  // namespace

// SphericalEikonal.Relax (SphericalEikonal.cs:284-325) with SettleTolerance 1e-7 and SweepRoundCap.
std::vector<double> relax_for_selftest(const Grid& g, const double* slow, const std::vector<int32_t>& seed_idx,
                                       const std::vector<double>& seed_t) {
    Metric m(g);
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    std::vector<double> a(size_t(g.count()), kInf);
    std::vector<uint8_t> fixed(a.size(), 0);
    for (size_t q = 0; q < seed_idx.size(); q++) {
        a[seed_idx[q]] = std::min(a[seed_idx[q]], seed_t[q]);
        fixed[seed_idx[q]] = 1;
    }
    const int cap = std::max(32, (nx + ny + nz) / 4);
    for (int phase = 0; phase < 2; phase++)
        for (int round = 0; round < cap; round++) {
            bool changed = false;
            for (int dir = 0; dir < 8; dir++)
                for (int p = 0; p < nx + ny + nz - 2; p++) {
                    int i0 = std::max(0, p - (ny - 1) - (nz - 1)), i1 = std::min(nx - 1, p);
                    int k0 = std::max(0, p - (nx - 1) - (ny - 1)), k1 = std::min(nz - 1, p);
                    for (int kp = k0; kp <= k1; kp++)
                        for (int ip = i0; ip <= i1; ip++) {
                            int jp = p - ip - kp;
                            if (jp < 0 || jp >= ny) continue;
                            int i = (dir & 1) ? nx - 1 - ip : ip;
                            int j = (dir & 2) ? ny - 1 - jp : jp;
                            int k = (dir & 4) ? nz - 1 - kp : kp;
                            int idx = g.index(i, j, k);
                            if (fixed[idx]) continue;
                            double cur = a[idx];
                            double cand = relax_node(g, m, slow, a.data(), idx, i, j, k, phase == 1);
                            if (!(cand < cur)) continue;
                            a[idx] = cand;
                            if (!std::isfinite(cur) || cur - cand > 1e-7) changed = true;
                        }
                }
            if (!changed) break;
        }
    return a;
}

}  // namespace host
}  // namespace ts
