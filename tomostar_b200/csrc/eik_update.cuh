// The upwind (Godunov) update of one eikonal node on the sphere, for both precisions.
//
// FP64: the reference arithmetic term for term — Forward/SphericalEikonal.cs:349-396 (RelaxNode)
// and Forward/EikonalOpenCl.cs:432-450, 560-599 (eik_axis, eik_sweep under QV_FP64). Every
// operation is an explicit round-to-nearest intrinsic, so the compiler can neither contract a
// multiply-add nor reorder: a result is the host's to the last bit, whichever kernel inlines it.
//
// FP32: the times are stored as float, and the update is solved as offsets from the smallest
// upwind neighbour r (the scheme of the reference's paired-float kernel, EikonalOpenCl.cs:484-497,
// 568-606): every quantity of the quadratic is then a cell crossing time, not an absolute time,
// so float keeps the digits that survive the discriminant's subtraction. The stored time is
// r + root rounded once to float.
//
// Extension (variable vertical spacing): the z axis may carry per-level coefficients instead of
// the uniform spacing; see zcoef_* below. A uniform grid never takes that path.
#pragma once

#include "ts_common.cuh"

namespace ts {

// Per-level coefficients of a non-uniform z axis, 16 per level k:
//   [0..7]  minus side (first neighbour k-1, second k-2): w1, w2, a, b, c, c/a, -, -
//   [8..15] plus side  (first neighbour k+1, second k+2): w1, w2, a, b, c, c/a, -, -
// with the one-sided three-point derivative a·T0 − b·T1 + c·T2, a = (2h1+h2)/(h1(h1+h2)),
// b = (h1+h2)/(h1 h2), c = h1/(h2(h1+h2)) (h1 = spacing to the first neighbour, h2 from there to
// the second), w1 = 1/(h1·h1) the first-order weight and w2 = 1/((1/a)·(1/a)) the second-order one.
// Uniform spacing gives a = 3/(2h), b = 2/h, c = 1/(2h): the reference's (4T1 − T2)/3 and 2h/3.
constexpr int kZCoef = 16;

// The weights of an axis term are precomputed per axis and level on the host with the reference's
// own operations (w1 = 1.0 / (h * h), w2 = 1.0 / (he * he) with he = 2 * h / 3;
// SphericalEikonal.cs:369, 391), so they are the same bits the reference divides out per update.

// ---- FP64, exact --------------------------------------------------------------------------------

TS_DEVINL double dmul(double a, double b) { return __dmul_rn(a, b); }
TS_DEVINL double dadd(double a, double b) { return __dadd_rn(a, b); }
TS_DEVINL double dsub(double a, double b) { return __dadd_rn(a, -b); }
TS_DEVINL double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// a / 3 correctly rounded, for finite a >= 0 (the reference's (4·first − t2)/3, t2 <= first):
// q0 = RN(a·RN(1/3)) is within an ulp of a/3, r = a − 3·q0 is exact (FMA), and RN(q0 + r·RN(1/3))
// is the correctly rounded quotient because a/3 is never within a sixth of an ulp of a rounding
// midpoint (its fraction in half-ulps is 0, 1/3 or 2/3) while q0 + r·RN(1/3) is within 2^-50 ulp of
// a/3. Same bits as __ddiv_rn(a, 3.0), in three instructions.
TS_DEVINL double ddiv3(double a) {
    const double third = 0.33333333333333331;  // RN(1/3)
    double q0 = __dmul_rn(a, third);
    double r = __fma_rn(-3.0, q0, a);
    return __fma_rn(r, third, q0);
}

// One axis's term (SphericalEikonal.cs:381-395): the smaller neighbour, promoted to second order
// when its partner beyond is finite and not larger. Produces (effective time, weight, neighbour
// time); unused terms keep t = +inf and sort last.
template <bool VARZ>
TS_DEVINL void axis64(double minus, double plus, double minus2, double plus2, double w1, double w2, const double* zc,
                      bool second, double& te, double& we, double& tn, int& used) {
    double first, t2;
    bool minus_side = minus <= plus;
    if (minus_side) { first = minus; t2 = minus2; }
    else { first = plus; t2 = plus2; }
    if (!(first <= 1.7976931348623157e308)) return;  // not finite (first is never NaN)
    bool promote = second && (t2 <= 1.7976931348623157e308) && t2 <= first;
    if (!VARZ) {
        if (promote) { te = ddiv3(dsub(dmul(4.0, first), t2)); we = w2; }
        else { te = first; we = w1; }
    } else {
        const double* c = zc + (minus_side ? 0 : 8);
        if (promote) { te = ddiv(dsub(dmul(c[3], first), dmul(c[4], t2)), c[2]); we = c[1]; }
        else { te = first; we = c[0]; }
    }
    tn = first;
    used++;
}

// Stable sort of three (t, h, n) by t (SphericalEikonal.cs:246-254, 262-275).
template <typename R>
TS_DEVINL void sort3(R* t, R* h, R* n) {
    auto sw = [&](int a, int b) {
        R x = t[a]; t[a] = t[b]; t[b] = x;
        x = h[a]; h[a] = h[b]; h[b] = x;
        x = n[a]; n[a] = n[b]; n[b] = x;
    };
    if (t[0] > t[1]) sw(0, 1);
    if (t[1] > t[2]) {
        sw(1, 2);
        if (t[0] > t[1]) sw(0, 1);
    }
}

// The Godunov root over the first `terms` sorted terms; false when the discriminant is negative
// or the root falls below a neighbour it used (SphericalEikonal.cs:364-378).
TS_DEVINL bool root64(int terms, const double* t, const double* w, const double* n, double s, double& root) {
    double sw = 0.0, swt = 0.0, swt2 = 0.0;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        if (r < terms) {
            sw = dadd(sw, w[r]);
            swt = dadd(swt, dmul(w[r], t[r]));
            swt2 = dadd(swt2, dmul(dmul(w[r], t[r]), t[r]));
        }
    }
    double disc = dsub(dmul(swt, swt), dmul(sw, dsub(swt2, dmul(s, s))));
    if (disc < 0.0) return false;
    root = ddiv(dadd(swt, __dsqrt_rn(disc)), sw);
#pragma unroll
    for (int r = 0; r < 3; r++)
        if (r < terms && root < n[r]) return false;
    return true;
}

// RelaxNode (SphericalEikonal.cs:349-379): the candidate time of a node from its 12 neighbour
// values (+inf off the grid). xm/xp = i∓1, xm2/xp2 = i∓2, likewise y and z; (w1, w2) are each
// axis's first- and second-order weights.
template <bool VARZ>
TS_DEVINL double update64(double s, double xm, double xp, double xm2, double xp2, double ym, double yp, double ym2,
                          double yp2, double zm, double zp, double zm2, double zp2, double wx1, double wx2,
                          double wy1, double wy2, double wz1, double wz2, const double* zc, bool second) {
    const double inf = dinf();
    if (!(s > 0.0)) return inf;
    double t[3] = {inf, inf, inf}, w[3] = {1.0, 1.0, 1.0}, n[3] = {inf, inf, inf};
    int used = 0;
    axis64<false>(xm, xp, xm2, xp2, wx1, wx2, nullptr, second, t[0], w[0], n[0], used);
    axis64<false>(ym, yp, ym2, yp2, wy1, wy2, nullptr, second, t[1], w[1], n[1], used);
    axis64<VARZ>(zm, zp, zm2, zp2, wz1, wz2, zc, second, t[2], w[2], n[2], used);
    if (used == 0) return inf;
    sort3(t, w, n);
    double root;
    if (used >= 3 && root64(3, t, w, n, s, root)) return root;
    if (used >= 2 && root64(2, t, w, n, s, root)) return root;
    if (root64(1, t, w, n, s, root)) return root;
    return inf;
}

// ---- FP32, offsets from the smallest upwind neighbour -------------------------------------------

// Explicit intrinsics here too, so that two kernels inlining this update round identically.
TS_DEVINL float fmul(float a, float b) { return __fmul_rn(a, b); }
TS_DEVINL float fadd(float a, float b) { return __fadd_rn(a, b); }
TS_DEVINL float fsub(float a, float b) { return __fadd_rn(a, -b); }
TS_DEVINL float fdiv(float a, float b) { return __fdiv_rn(a, b); }
TS_DEVINL float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

struct Pick32 {
    float first, t2;
    bool minus_side, ok;
};

TS_DEVINL Pick32 pick32(float minus, float plus, float minus2, float plus2) {
    Pick32 p;
    p.minus_side = minus <= plus;
    p.first = p.minus_side ? minus : plus;
    p.t2 = p.minus_side ? minus2 : plus2;
    p.ok = p.first <= 3.4028234663852886e38f;
    return p;
}

template <bool VARZ>
TS_DEVINL void term32(const Pick32& p, float r, float w1, float w2, const float* zc, bool second, float& te, float& we,
                      float& tn) {
    float of = fsub(p.first, r);
    bool promote = second && (p.t2 <= 3.4028234663852886e38f) && p.t2 <= p.first;
    if (!VARZ) {
        if (promote) { te = ffma(fsub(p.first, p.t2), 0.333333343f, of); we = w2; }
        else { te = of; we = w1; }
    } else {
        const float* c = zc + (p.minus_side ? 0 : 8);
        if (promote) { te = ffma(fsub(p.first, p.t2), c[5], of); we = c[1]; }
        else { te = of; we = c[0]; }
    }
    tn = of;
}

TS_DEVINL bool root32(int terms, const float* t, const float* w, const float* n, float s, float& root) {
    float base = t[0];
    float sw = 0.f, swd = 0.f, swd2 = 0.f;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        if (r < terms) {
            float d = fsub(t[r], base);
            sw = fadd(sw, w[r]);
            float wd = fmul(w[r], d);
            swd = fadd(swd, wd);
            swd2 = ffma(wd, d, swd2);
        }
    }
    float disc = ffma(swd, swd, -fmul(sw, ffma(-s, s, swd2)));
    if (disc < 0.f) return false;
    root = fadd(base, fdiv(fadd(swd, __fsqrt_rn(disc)), sw));
#pragma unroll
    for (int r = 0; r < 3; r++)
        if (r < terms && root < n[r]) return false;
    return true;
}

// The FP32 candidate time of a node (same inputs as update64).
template <bool VARZ>
TS_DEVINL float update32(float s, float xm, float xp, float xm2, float xp2, float ym, float yp, float ym2, float yp2,
                         float zm, float zp, float zm2, float zp2, float wx1, float wx2, float wy1, float wy2,
                         float wz1, float wz2, const float* zc, bool second) {
    const float inf = real_inf<float>();
    if (!(s > 0.f)) return inf;
    Pick32 px = pick32(xm, xp, xm2, xp2), py = pick32(ym, yp, ym2, yp2), pz = pick32(zm, zp, zm2, zp2);
    int used = int(px.ok) + int(py.ok) + int(pz.ok);
    if (used == 0) return inf;
    float r = fminf(px.ok ? px.first : inf, fminf(py.ok ? py.first : inf, pz.ok ? pz.first : inf));
    float t[3] = {inf, inf, inf}, w[3] = {1.f, 1.f, 1.f}, n[3] = {inf, inf, inf};
    if (px.ok) term32<false>(px, r, wx1, wx2, nullptr, second, t[0], w[0], n[0]);
    if (py.ok) term32<false>(py, r, wy1, wy2, nullptr, second, t[1], w[1], n[1]);
    if (pz.ok) term32<VARZ>(pz, r, wz1, wz2, zc, second, t[2], w[2], n[2]);
    sort3(t, w, n);
    float root;
    bool found = (used >= 3 && root32(3, t, w, n, s, root)) || (used >= 2 && root32(2, t, w, n, s, root)) ||
                 root32(1, t, w, n, s, root);
    return found ? fadd(r, root) : inf;
}

// Generic front ends used by the kernels.
template <typename Real, bool VARZ>
struct Update;

template <bool VARZ>
struct Update<double, VARZ> {
    TS_DEVINL static double eval(double s, double xm, double xp, double xm2, double xp2, double ym, double yp,
                                 double ym2, double yp2, double zm, double zp, double zm2, double zp2, double wx1,
                                 double wx2, double wy1, double wy2, double wz1, double wz2, const double* zc,
                                 bool second) {
        return update64<VARZ>(s, xm, xp, xm2, xp2, ym, yp, ym2, yp2, zm, zp, zm2, zp2, wx1, wx2, wy1, wy2, wz1, wz2,
                              zc, second);
    }
};

template <bool VARZ>
struct Update<float, VARZ> {
    TS_DEVINL static float eval(float s, float xm, float xp, float xm2, float xp2, float ym, float yp, float ym2,
                                float yp2, float zm, float zp, float zm2, float zp2, float wx1, float wx2, float wy1,
                                float wy2, float wz1, float wz2, const float* zc, bool second) {
        return update32<VARZ>(s, xm, xp, xm2, xp2, ym, yp, ym2, yp2, zm, zp, zm2, zp2, wx1, wx2, wy1, wy2, wz1, wz2,
                              zc, second);
    }
};

// Whether a drop wakes the node's stencil neighbours: every drop when wake_rel is 0 (the reference),
// otherwise a drop larger than wake_rel × the new time (or from +inf).
template <typename Real>
TS_DEVINL bool wakes(Real cur, Real cand, Real wake_rel);
template <>
TS_DEVINL bool wakes<double>(double cur, double cand, double wake_rel) {
    return !(cur <= 1.7976931348623157e308) || dsub(cur, cand) > dmul(wake_rel, cand);
}
template <>
TS_DEVINL bool wakes<float>(float cur, float cand, float wake_rel) {
    return !(cur <= 3.4028234663852886e38f) || fsub(cur, cand) > fmul(wake_rel, cand);
}

// Whether a drop counts towards "the round changed something" (SphericalEikonal.cs:319).
template <typename Real>
TS_DEVINL bool counts_as_change(Real cur, Real cand, Real tol) {
    return !(cur <= Real(3.4028234663852886e38)) || (cur - cand) > tol;
}
template <>
TS_DEVINL bool counts_as_change<double>(double cur, double cand, double tol) {
    return !(cur <= 1.7976931348623157e308) || dsub(cur, cand) > tol;
}

}  // namespace ts
