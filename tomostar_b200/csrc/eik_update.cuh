// The upwind (Godunov) update of one eikonal node on the sphere, for both precisions.
//
// FP64: the reference arithmetic term for term — Forward/SphericalEikonal.cs:349-396 (RelaxNode)
// and Forward/EikonalOpenCl.cs:432-450, 560-599 (eik_axis, eik_sweep under QV_FP64). Every
// operation is an explicit round-to-nearest intrinsic, so the compiler can neither contract a
// multiply-add nor reorder: a result is the host's to the last bit, whichever kernel inlines it.
//
// FP32: the reference's paired-float kernel (times as hi + lo float pairs, the update in float
// offsets from the smallest upwind neighbour; EikonalOpenCl.cs:454-497, 545-606), term for term.
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

// The Godunov root over the first `terms` sorted terms (SphericalEikonal.cs:364-378). The reference
// adds the terms in sorted order, so the sums of k terms are the running sums after the k-th term:
// they are formed once and a retry with one term fewer reuses them (same operations, same bits).
struct Sums64 {
    double sw, swt, swt2;
};

TS_DEVINL Sums64 add_term(Sums64 q, double w, double t) {
    q.sw = dadd(q.sw, w);
    q.swt = dadd(q.swt, dmul(w, t));
    q.swt2 = dadd(q.swt2, dmul(dmul(w, t), t));
    return q;
}

// The candidate of `terms` terms from their sums; false when the discriminant is negative or the root
// falls below a neighbour it used.
TS_DEVINL bool root_from(const Sums64& q, int terms, const double* n, double s, double& root) {
    const double disc = dsub(dmul(q.swt, q.swt), dmul(q.sw, dsub(q.swt2, dmul(s, s))));
    if (disc < 0.0) return false;
    root = ddiv(dadd(q.swt, __dsqrt_rn(disc)), q.sw);
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
    const Sums64 q1 = add_term(Sums64{0.0, 0.0, 0.0}, w[0], t[0]);
    const Sums64 q2 = add_term(q1, w[1], t[1]);
    const Sums64 q3 = add_term(q2, w[2], t[2]);
    double root;
    if (used >= 3 && root_from(q3, 3, n, s, root)) return root;
    if (used >= 2 && root_from(q2, 2, n, s, root)) return root;
    if (root_from(q1, 1, n, s, root)) return root;
    return inf;
}

// ---- FP32: times as float pairs hi + lo, the update in float offsets -----------------------------
//
// The reference's paired-float kernel term for term (EikonalOpenCl.cs:454-497 df_sub, df_add,
// df_less, eik_pick, eik_term; 545-606 the root and the acceptance): each axis's upwind neighbour is
// chosen by the lexicographic order of (hi, lo), the reference time r is the smallest of them, every
// term is a float offset from r (a cell crossing time, so float keeps the digits that survive the
// discriminant's subtraction), and the result r + root is formed as a pair by Knuth's two-sum.
// Every float operation is an explicit round-to-nearest intrinsic (the kernel's FP_CONTRACT OFF),
// so the result equals the reference kernel's to the bit on the same inputs.

TS_DEVINL float fmul(float a, float b) { return __fmul_rn(a, b); }
TS_DEVINL float fadd(float a, float b) { return __fadd_rn(a, b); }
TS_DEVINL float fsub(float a, float b) { return __fadd_rn(a, -b); }
TS_DEVINL float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// df_sub: (a.hi − b.hi) + (a.lo − b.lo).
TS_DEVINL float psub(Pair a, Pair b) { return fadd(fsub(a.hi, b.hi), fsub(a.lo, b.lo)); }
// df_less: lexicographic on (hi, lo).
TS_DEVINL bool pless(Pair a, Pair b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
// df_add: r + x as hi + lo (Knuth's two-sum of r.hi and r.lo + x).
TS_DEVINL Pair padd(Pair r, float x) {
    float b = fadd(r.lo, x);
    float s = fadd(r.hi, b);
    float bb = fsub(s, r.hi);
    float e = fadd(fsub(r.hi, fsub(s, bb)), fsub(b, bb));
    return Pair(s, e);
}

struct PickP {
    Pair first, t2;
    bool minus_side, ok;
};

// eik_pick: the upwind neighbour of one axis and its second-order partner (+inf when absent or when
// the update is first order: the kernels pass +inf for nodes off the grid).
TS_DEVINL PickP pickp(Pair minus, Pair plus, Pair minus2, Pair plus2) {
    PickP p;
    p.minus_side = !pless(plus, minus);
    p.first = p.minus_side ? minus : plus;
    p.t2 = p.minus_side ? minus2 : plus2;
    p.ok = finite_r(p.first.hi);
    return p;
}

// eik_term: the axis's term as offsets from r. Extension (variable depth spacing): the second-order
// term takes the level's coefficient c/a in place of 1/3.
template <bool VARZ>
TS_DEVINL void termp(const PickP& p, Pair r, float w1, float w2, const Pair* zc, bool second, float& te, float& we,
                     float& tn) {
    const float of = psub(p.first, r);
    const bool promote = second && finite_r(p.t2.hi) && !pless(p.first, p.t2);
    if (!VARZ) {
        if (promote) { te = fadd(of, fdiv(psub(p.first, p.t2), 3.0f)); we = w2; }
        else { te = of; we = w1; }
    } else {
        const Pair* c = zc + (p.minus_side ? 0 : 8);
        if (promote) { te = fadd(of, fmul(psub(p.first, p.t2), c[5].hi)); we = c[1].hi; }
        else { te = of; we = c[0].hi; }
    }
    tn = of;
}

// The root over the first `terms` sorted terms, as offsets from base = te[0] (EikonalOpenCl.cs:575-597).
TS_DEVINL bool rootp(int terms, const float* t, const float* w, const float* n, float s, float& root) {
    const float base = t[0];
    float sw = 0.f, swd = 0.f, swd2 = 0.f;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        if (q < terms) {
            const float d = fsub(t[q], base);
            sw = fadd(sw, w[q]);
            swd = fadd(swd, fmul(w[q], d));
            swd2 = fadd(swd2, fmul(fmul(w[q], d), d));
        }
    }
    const float disc = fsub(fmul(swd, swd), fmul(sw, fsub(swd2, fmul(s, s))));
    if (disc < 0.f) return false;
    root = fadd(base, fdiv(fadd(swd, __fsqrt_rn(disc)), sw));
#pragma unroll
    for (int q = 0; q < 3; q++)
        if (q < terms && root < n[q]) return false;
    return true;
}

// The paired candidate time of a node (same inputs as update64; slowness and weights in hi).
template <bool VARZ>
TS_DEVINL Pair updatep(Pair sp, Pair xm, Pair xp, Pair xm2, Pair xp2, Pair ym, Pair yp, Pair ym2, Pair yp2, Pair zm,
                       Pair zp, Pair zm2, Pair zp2, Pair wx1, Pair wx2, Pair wy1, Pair wy2, Pair wz1, Pair wz2,
                       const Pair* zc, bool second) {
    const Pair inf = real_inf<Pair>();
    const float s = sp.hi;
    if (!(s > 0.f)) return inf;
    const Pair pinf = inf;
    PickP px = pickp(xm, xp, second ? xm2 : pinf, second ? xp2 : pinf);
    PickP py = pickp(ym, yp, second ? ym2 : pinf, second ? yp2 : pinf);
    PickP pz = pickp(zm, zp, second ? zm2 : pinf, second ? zp2 : pinf);
    if (!(px.ok || py.ok || pz.ok)) return inf;
    Pair r = inf;
    if (px.ok && pless(px.first, r)) r = px.first;
    if (py.ok && pless(py.first, r)) r = py.first;
    if (pz.ok && pless(pz.first, r)) r = pz.first;
    const float finf = __builtin_huge_valf();
    float t[3] = {finf, finf, finf}, w[3] = {1.f, 1.f, 1.f}, n[3] = {finf, finf, finf};
    int used = 0;
    if (px.ok) { termp<false>(px, r, wx1.hi, wx2.hi, nullptr, second, t[0], w[0], n[0]); used++; }
    if (py.ok) { termp<false>(py, r, wy1.hi, wy2.hi, nullptr, second, t[1], w[1], n[1]); used++; }
    if (pz.ok) { termp<VARZ>(pz, r, wz1.hi, wz2.hi, zc, second, t[2], w[2], n[2]); used++; }
    sort3(t, w, n);
    float root;
    const bool found = (used >= 3 && rootp(3, t, w, n, s, root)) || (used >= 2 && rootp(2, t, w, n, s, root)) ||
                       rootp(1, t, w, n, s, root);
    if (!found || !finite_r(root)) return inf;
    return padd(r, root);
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
struct Update<Pair, VARZ> {
    TS_DEVINL static Pair eval(Pair s, Pair xm, Pair xp, Pair xm2, Pair xp2, Pair ym, Pair yp, Pair ym2, Pair yp2,
                               Pair zm, Pair zp, Pair zm2, Pair zp2, Pair wx1, Pair wx2, Pair wy1, Pair wy2, Pair wz1,
                               Pair wz2, const Pair* zc, bool second) {
        return updatep<VARZ>(s, xm, xp, xm2, xp2, ym, yp, ym2, yp2, zm, zp, zm2, zp2, wx1, wx2, wy1, wy2, wz1, wz2,
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
TS_DEVINL bool wakes<Pair>(Pair cur, Pair cand, Pair wake_rel) {
    return !finite_r(cur.hi) || psub(cur, cand) > fmul(wake_rel.hi, cand.hi);
}

// Whether a drop counts towards "the round changed something" (SphericalEikonal.cs:319; the paired
// kernel's `drop > TOL`, EikonalOpenCl.cs:604).
template <typename Real>
TS_DEVINL bool counts_as_change(Real cur, Real cand, Real tol);
template <>
TS_DEVINL bool counts_as_change<double>(double cur, double cand, double tol) {
    return !(cur <= 1.7976931348623157e308) || dsub(cur, cand) > tol;
}
template <>
TS_DEVINL bool counts_as_change<Pair>(Pair cur, Pair cand, Pair tol) {
    return psub(cur, cand) > tol.hi;
}

}  // namespace ts
