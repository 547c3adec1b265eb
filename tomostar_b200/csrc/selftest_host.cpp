// The self-test gates' host solvers (EikonalOpenCl.SelfTest compares the device with
// SphericalEikonal.Relax on the host, Forward/EikonalOpenCl.cs:346-374; LsqrOpenCl.SelfTest with
// Lsqr.Solve, Numerics/LsqrOpenCl.cs:541-557). Used by ts_cuda_selftest and ts_lsqr_selftest only;
// no solve ever returns their results. Compiled with -ffp-contract=off.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

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

// Lsqr.Solve (Numerics/Lsqr.cs:33-152), sequential, for LsqrOpenCl.SelfTest's host side
// (Numerics/LsqrOpenCl.cs:541-557). Returns the iteration count; x has n entries.
int lsqr_for_selftest(int m, int n, const int32_t* rp, const int32_t* ci, const double* va, const double* b,
                      double damp, int max_it, double atol, double btol, double conlim, double* x) {
    const size_t nn = static_cast<size_t>(n);
    std::vector<double> u(b, b + m), v(nn, 0.0), w(nn, 0.0), tn(nn, 0.0);
    std::fill(x, x + n, 0.0);
    auto norm = [](const std::vector<double>& a) {
        double s = 0;
        for (double e : a) s += e * e;
        return std::sqrt(s);
    };
    auto scale = [](std::vector<double>& a, double f) {
        for (double& e : a) e *= f;
    };
    auto atx = [&](const std::vector<double>& in, std::vector<double>& out) {  // out = Aᵀ in
        std::fill(out.begin(), out.end(), 0.0);
        for (int i = 0; i < m; i++)
            for (int e = rp[i]; e < rp[i + 1]; e++) out[ci[e]] += va[e] * in[i];
    };
    double beta = norm(u);
    if (beta == 0) return 0;
    const double bnorm = beta;
    scale(u, 1.0 / beta);
    atx(u, v);
    double alpha = norm(v);
    if (alpha == 0) return 0;
    scale(v, 1.0 / alpha);
    w = v;
    double rhobar = alpha, phibar = beta, ddnorm = 0, xxnorm = 0, z = 0, cs2 = -1, sn2 = 0, anorm2 = 0, damped2 = 0;
    const double ctol = conlim > 0 ? 1.0 / conlim : 0.0;
    int it = 0;
    while (it < max_it) {
        it++;
        for (int i = 0; i < m; i++) {
            double acc = 0;
            for (int e = rp[i]; e < rp[i + 1]; e++) acc += va[e] * v[ci[e]];
            u[i] = acc - alpha * u[i];
        }
        beta = norm(u);
        if (beta > 0) {
            scale(u, 1.0 / beta);
            anorm2 += alpha * alpha + beta * beta + damp * damp;
            atx(u, tn);
            for (int q = 0; q < n; q++) v[q] = tn[q] - beta * v[q];
            alpha = norm(v);
            if (alpha > 0) scale(v, 1.0 / alpha);
        }
        const double rhobar1 = std::sqrt(rhobar * rhobar + damp * damp);
        const double cs1 = rhobar / rhobar1, sn1 = damp / rhobar1, psi = sn1 * phibar;
        phibar = cs1 * phibar;
        const double rho = std::sqrt(rhobar1 * rhobar1 + beta * beta);
        const double cs = rhobar1 / rho, sn = beta / rho, theta = sn * alpha;
        rhobar = -cs * alpha;
        const double phi = cs * phibar;
        phibar = sn * phibar;
        const double tau = sn * phi;
        double ww = 0;
        for (double e : w) ww += e * e;
        ddnorm += ww / (rho * rho);
        for (int q = 0; q < n; q++) {
            x[q] += phi / rho * w[q];
            w[q] = v[q] - theta / rho * w[q];
        }
        const double delta = sn2 * rho, gambar = -cs2 * rho, rhs = phi - delta * z;
        const double gamma = std::sqrt(gambar * gambar + theta * theta);
        cs2 = gambar / gamma;
        sn2 = theta / gamma;
        z = rhs / gamma;
        xxnorm += z * z;
        damped2 += psi * psi;
        const double anorm = std::sqrt(anorm2), acond = anorm * std::sqrt(ddnorm), arnorm = alpha * std::fabs(tau);
        const double rnorm = std::sqrt(phibar * phibar + damped2), xnorm = std::sqrt(xxnorm);
        const double test1 = rnorm / bnorm, test2 = arnorm / std::max(1e-300, anorm * rnorm);
        const double test3 = 1.0 / std::max(1e-300, acond), t1 = test1 / (1 + anorm * xnorm / bnorm);
        const double rtol = btol + atol * anorm * xnorm / bnorm;
        if (test1 <= rtol || test2 <= atol || (ctol > 0 && test3 <= ctol) || 1 + t1 <= 1 || 1 + test2 <= 1 ||
            1 + test3 <= 1 || beta == 0 || alpha == 0)
            break;
    }
    return it;
}

}  // namespace host
}  // namespace ts
