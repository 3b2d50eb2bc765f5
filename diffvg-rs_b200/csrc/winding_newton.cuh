// winding_newton.cuh — the winding contribution of a cubic segment without the f64
// transcendental functions of the crate's root formula, whenever it provably comes out
// the same.
//
// The crate decides a cubic segment's crossings of the +x ray from (px, py) with the f64
// roots of y(t) = py from solve_cubic (src/distance/curve.rs / winding.rs:170-192): the
// normalised cubic t^3 + b t^2 + c t + d, q = (b^2 - 3c)/9, r = (2b^3 - 9bc + 27d)/54,
// three roots t_k = -2 sqrt(q) cos((acos(r / sqrt(q^3)) + 2 pi k) / 3) - b/3 when
// r^2 < q^3, else one root (Cardano: ar = -sign(r) cbrt(|r| + sqrt(r^2 - q^3)),
// t = ar + q/ar - b/3).  Each root in [0, 1] whose x(t) lies right of px adds the sign
// of y'(t).
//
// Here q and r (and the branch) are computed exactly as the crate computes them; the
// roots y_k = t_k + b/3 of g(y) = y^3 - 3 q y + 2 r, the exact roots of the crate's own
// (rounded) q and r, are estimated in f32 and polished by one f64 Newton step.  Each
// polished root carries a bound on its distance to the exact root (Newton's quadratic
// convergence from a root known to lie within 2|step|, plus the rounding of the step)
// and the crate's computed root a bound on its own (the rounding of its formula, which
// grows as 1 / sqrt(1 - (r / sqrt(q^3))^2) near a double root and with the exponent
// rounding of pow(x, 1/3)).  A decision (t in [0, 1], x(t) > px, y'(t) > 0) is taken
// here only when it holds over the union of both bounds and the rounding of the crate's
// evaluations; otherwise the caller runs the crate's formula.  The f64 acos and three f64
// cos of the three-root branch (and the f64 pow of the one-root branch) dominate the
// solve: one f64 division per root replaces them.
//
// Host and device share this code: the CPU stress harness (oracle/winding_stress.cpp)
// runs it against the oracle's restatement of the crate's f64 computation, with the f32
// estimates moved by a random amount to cover the device's fast cosine.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define DVG_WN_HD __host__ __device__ __forceinline__
#else
#define DVG_WN_HD inline
#endif

namespace dvgb {

constexpr int WIND_UNSURE = 0x7fff;
constexpr double WN_EPS = 1.1102230246251565e-16;  // 2^-53

DVG_WN_HD float wn_cos(float x) {
#ifdef __CUDA_ARCH__
    return __cosf(x);
#else
    return std::cos(x);
#endif
}
DVG_WN_HD float wn_rsqrt(float x) {
#ifdef __CUDA_ARCH__
    return rsqrtf(x);
#else
    return 1.0f / std::sqrt(x);
#endif
}
// a / b for the error bounds (within 2 ulp on the device; every bound carries slack)
DVG_WN_HD float wn_div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
// |binary exponent| + 1 of a normal positive float: log2 bound for |ln x|
DVG_WN_HD float wn_log2_bound(float x) {
#ifdef __CUDA_ARCH__
    const int e = ((__float_as_int(x) >> 23) & 255) - 127;
#else
    const int e = std::ilogb(x);
#endif
    return (float)((e < 0 ? -e : e) + 1);
}

// One Newton step on g(y) = y^3 - 3 q y + 2 r from the f32 estimate y0 (f64 residual, f32
// reciprocal of g': the correction needs only its own relative accuracy).  Returns the new
// root; *u (f32) bounds its distance to the exact root of g within 2|step| of y0, which
// exists and is unique when h = |g''| |step| / |g'(y0)| <= 1/4 (Kantorovich: <= 1/2);
// then Newton's error is at most (|g''| / (2|g'|)) (2|step|)^2 = 2 h |step|.  *u < 0: no
// bound.  q3x = 3q, r2x = 2r, aqr = 3|q| and 2|r| for the residual's rounding.
DVG_WN_HD double wn_newton(float y0f, double q3x, double r2x, double q, float aq3, float ar2, float dq, float dr,
                           float* u) {
    const double y0 = (double)y0f;
    const double y2 = y0 * y0;
    const double g = (y2 - q3x) * y0 + r2x;
    const float gp = 3.0f * (y0f * y0f - (float)q);
    const float ag = std::fabs(gp);
    if (!(ag > 1.0e-30f && ag < 1.0e30f)) {
        *u = -1.0f;
        return y0;
    }
    const float inv = wn_div(1.0f, gp);
    const double s = g * (double)inv;
    const double y1 = y0 - s;
    const float as = (float)std::fabs(s), ai = std::fabs(inv), ay = std::fabs(y0f);
    // |g''| = |6y| within 2|s| of y0; g' from f32 (its rounding, ~1e-6 of |g'| once the
    // 1/4 margin below holds, is inside the slack)
    const float h = 6.0f * (ay + 2.0f * as) * as * ai * 1.01f;
    if (!(h <= 0.25f)) {
        *u = -1.0f;
        return y1;
    }
    const float gabs = (ay * ay + aq3) * ay + ar2;
    // Newton + the f64 residual's rounding + the f32 reciprocal's (2 ulp + the f32 g') + the
    // update's rounding
    // + the distance to the root of the crate's g (its q and r differ by dq, dr): twice the
    // first-order shift, g' varying by less than half over the ball
    *u = (2.0f * h * as + (16.0f * (float)WN_EPS * gabs + 2.0f * (3.0f * ay * dq + 2.0f * dr)) * ai + as * 2.5e-6f +
          8.0f * (float)WN_EPS * ay) * 1.01f;
    return y1;
}

// The crate's decision for one root y (+ its bound uy) of the normalised cubic, t = y - b3
// (b3 = the crate's b/3): 0 (no crossing counted), +-1, or WIND_UNSURE.  a..c: y(t)
// coefficients as the crate forms them; ax..dx: x(t) - px.  For t in [0, 1 + 1e-3]:
// |d/dt (x(t) - px)| <= 3|ax| T^2 + 2|bx| T + |cx| and the crate's and our evaluations of
// x(t) - px each within 8 eps of the sum of |terms|; the same for y'(t) = 3a t^2 + 2b t + c
// (derivative 6|a| T + 2|b|).
DVG_WN_HD int wn_decide(double y, float uy, double b3, double a, double b, double c, double ax, double bx, double cx,
                        double dx) {
    const double t = y - b3;
    // the crate's t = fl(y_crate - b3) against ours: both roots' bounds and both roundings
    const double ut = ((double)uy + 4.5e-16 * std::fabs(y) + 9.0e-16 * std::fabs(b3)) * 1.001;
    if (!(ut < 1.0e-3)) return WIND_UNSURE;
    if (t + ut < 0.0 || t - ut > 1.0) return 0;  // outside [0, 1] for both
    if (!(t - ut >= 0.0 && t + ut <= 1.0)) return WIND_UNSURE;
    // x(t) - px = ax t^3 + bx t^2 + cx t + dx, the crate's evaluation order
    const double tp = ax * t * t * t + bx * t * t + cx * t + dx;
    const double fax = std::fabs(ax), fbx = std::fabs(bx), fcx = std::fabs(cx);
    const double mx = (3.02 * fax + 2.01 * fbx + fcx) * ut + 2.5e-15 * (fax + fbx + fcx + std::fabs(dx));
    if (!(std::fabs(tp) > mx)) return WIND_UNSURE;
    if (!(tp > 0.0)) return 0;
    // y'(t) = 3 a t^2 + 2 b t + c
    const double dy = 3.0 * a * t * t + 2.0 * b * t + c;
    const double fa = std::fabs(a), fb = std::fabs(b);
    const double my = (6.02 * fa + 2.01 * fb) * ut + 2.5e-15 * (3.01 * fa + 2.01 * fb + std::fabs(c));
    if (!(std::fabs(dy) > my)) return WIND_UNSURE;
    return dy > 0.0 ? 1 : -1;
}

// The roots of the crate's solve_cubic(a, b, c, d) that can fall in [0, 1], certified: for
// each of them, in the crate's order, per_root(y, uy, b3) with y a root of g and uy the
// bound on its distance to the crate's root (t = y - b3); roots whose estimate lies clearly
// outside [0, 1] are skipped.  Returns the sum of per_root's results, or WIND_UNSURE (also
// when per_root returns it).
// perturb: host stress harness only — each f32 estimate moves by perturb[k] times the
// scale of its formula (2 sqrt(q), or |ar| + |q / ar|).
// tight: bound the crate's three-root rounding from this cubic's 1 - x^2 (one more rsqrt)
// instead of its worst case 1e-6 (needed where the roots' f32 rounding must be certain).
template <bool tight = false, typename PerRoot>
DVG_WN_HD int cubic_roots_certified(double a, double b, double c, double d, PerRoot&& per_root,
                                    const float* perturb) {
    if (std::fabs(a) < 1.0e-6) return WIND_UNSURE;  // the crate's quadratic branch
    // The crate divides: b/a, c/a, d/a, /9, /54, /3.  One reciprocal and products give
    // values within a few eps of its own; g below has roots within dy of the crate's g (its
    // q and r), which the bounds carry (qa, ra: the sums of |terms| of q and r).
    const double ia = 1.0 / a;
    const double bn = b * ia, cn = c * ia, dn = d * ia;
    const double q = (bn * bn - 3.0 * cn) * (1.0 / 9.0);
    const double r = (2.0 * bn * bn * bn - 9.0 * bn * cn + 27.0 * dn) * (1.0 / 54.0);
    const double b3 = bn * (1.0 / 3.0);
    const double q3 = q * q * q, rr = r * r;
    const double q3x = 3.0 * q, r2x = 2.0 * r;
    const float aq3 = (float)std::fabs(q3x), ar2 = (float)std::fabs(r2x);
    if (!(aq3 < 1.0e30f && ar2 < 1.0e30f)) return WIND_UNSURE;
    // |our q - the crate's q| <= 16 eps (b^2 + 3|c|) / 9 + 3 eps |q| and |our r - the crate's r|
    // <= 19 eps (2|b|^3 + 9|b c| + 27|d|) / 54 + 3 eps |r| (inputs within 3 eps, both roundings),
    // taken with a margin of 2.5 or more
    float dq, dr;
    {
        const float fb = (float)std::fabs(bn), fc = (float)std::fabs(cn), fd = (float)std::fabs(dn);
        if (!(fb < 1.0e12f && fc < 1.0e24f && fd < 1.0e30f)) return WIND_UNSURE;
        dq = 2.0e-15f * (fb * fb + 3.0f * fc);
        dr = 1.0e-16f * ((2.0f * fb * fb + 9.0f * fc) * fb + 27.0f * fd) + 1.0e-15f * (float)std::fabs(r);
    }
    int w = 0;
    if (rr < q3) {  // three roots
        // 1 - x^2 >= 1e-6 for the crate's x = r / sqrt(q^3) (without its sqrt)
        if (!(q3 - rr >= 1.0e-6 * q3)) return WIND_UNSURE;  // near a double root
        const float sq = std::sqrt((float)q);
        if (!(sq > 1.0e-30f && sq < 1.0e12f)) return WIND_UNSURE;
        const float th = std::acos(std::fmin(std::fmax((float)r * wn_rsqrt((float)q3), -1.0f), 1.0f));
        // the crate's rounding: acos(x) within 4 eps / sqrt(1 - x^2) + 8 eps (<= 4008 eps) of
        // the exact angle (x carries the rounding of sqrt, q^3 and the division), the cosines
        // and products a few eps more; 2 sqrt(q) times that bounds its root, doubled.
        const float ec = tight ? 4.0f * sq * (float)WN_EPS *
                                     (8.2f * wn_rsqrt((float)(q3 - rr)) * ((float)q * sq) + 32.0f)
                               : 3.7e-12f * sq;
        // the f32 estimates: x within 5e-7 of its value (casts, rsqrt, product), acos within
        // 2 ulp, so the angle within 5e-4 (1 / sqrt(1 - x^2) <= 1e3), the cosine (fast, 2^-21
        // absolute) and sqrt(q) a little more: each estimate within 3.4e-4 sqrt(q) of the
        // crate's root of the same index; 2e-3 sqrt(q) allowed.  A root whose estimate lies
        // farther than that outside [0, 1] is outside for the crate too and needs no Newton step.
        const float e0 = 2.0e-3f * sq;
        const float fb3 = (float)b3;
        // g is monotone between its stationary points -sqrt(q), sqrt(q): the crate's roots
        // k = 0, 2, 1 are the one root in (-inf, -sqrt q), (-sqrt q, sqrt q), (sqrt q, inf);
        // a certified root strictly inside its interval is the crate's k-th root.
        const float lo = sq * (1.0f - 1.0e-6f), hi = sq * (1.0f + 1.0e-6f);
#pragma unroll 1
        for (int k = 0; k < 3; ++k) {
            const float phi = (th + (k == 0 ? 0.0f : (k == 1 ? 6.2831853f : -6.2831853f))) * (1.0f / 3.0f);
            float y0 = -2.0f * sq * wn_cos(phi);
            if (perturb) y0 += perturb[k] * 2.0f * sq;
            {
                const float t0 = y0 - fb3, e = e0 + 2.4e-7f * (std::fabs(y0) + std::fabs(fb3));
                if (t0 + e < 0.0f || t0 - e > 1.0f) continue;
            }
            float u;
            const double y = wn_newton(y0, q3x, r2x, q, aq3, ar2, dq, dr, &u);
            if (u < 0.0f) return WIND_UNSURE;
            const float uy = u + ec;
            const float yf = (float)y;
            const bool inside = k == 0 ? yf + uy < -hi : (k == 1 ? yf - uy > hi : std::fabs(yf) + uy < lo);
            if (!inside) return WIND_UNSURE;
            const int dk = per_root(y, uy, b3);
            if (dk == WIND_UNSURE) return WIND_UNSURE;
            w += dk;
        }
        return w;
    }
    // one root
    const double disc = rr - q3;
    const double s = std::sqrt(disc);
    const double m = std::fabs(r) + s;  // |cbrt argument| of the crate
    // the crate's s: sqrt of a difference carrying 3 eps (r^2 + |q^3|) of rounding, so within
    // 1.5 eps (r^2 + |q^3|) / (r^2 - q^3) of itself; kept below 1e-9 of s (so of m)
    if (!(3.0 * WN_EPS * (rr + std::fabs(q3)) < 1.0e-9 * s * s)) return WIND_UNSURE;
    const float rel_s = tight ? (float)(1.6 * WN_EPS * ((rr + std::fabs(q3)) / disc)) : 3.4e-10f;
    const float mf = (float)m;
    if (!(mf > 1.0e-30f && mf < 1.0e30f)) return WIND_UNSURE;
    const float arf = (r > 0.0 ? -1.0f : 1.0f) * std::cbrt(mf);
    if (!(std::fabs(arf) > 4.0e-6f)) return WIND_UNSURE;  // the crate's br = 0 branch nearby
    const float brf = wn_div((float)q, arf);
    float y0 = arf + brf;
    if (perturb) y0 += perturb[0] * (std::fabs(arf) + std::fabs(brf));
    float u;
    const double y = wn_newton(y0, q3x, r2x, q, aq3, ar2, dq, dr, &u);
    if (u < 0.0f) return WIND_UNSURE;
    // the crate's ar = +-pow(m, 1/3): the exponent's rounding (|ln m| eps / 3), pow's own
    // ulp and the error of s (rel_s of s, so of m; a third of that on ar); br = q / ar follows ar
    const float rel = (float)WN_EPS * (0.7f * wn_log2_bound(mf) + 16.0f) + rel_s;
    const float uy = u + 4.04f * (std::fabs(arf) + std::fabs(brf)) * rel;
    return per_root(y, uy, b3);
}

// The winding contribution of a cubic segment (the crate's decisions), or WIND_UNSURE.
DVG_WN_HD int winding_cubic_newton(double a, double b, double c, double d, double ax, double bx, double cx, double dx,
                                   const float* perturb = nullptr) {
    return cubic_roots_certified(
        a, b, c, d, [&](double y, float uy, double b3) { return wn_decide(y, uy, b3, a, b, c, ax, bx, cx, dx); },
        perturb);
}

// The crate's candidates of the closest point on a quadratic segment (closest_point_quadratic,
// curve.rs:26-78): the roots in [0, 1] of its stationarity cubic A t^3 + B t^2 + C t + D,
// as the f32 parameters t32 = (float)t the crate evaluates, in the crate's order.  Returns
// the count, or -1 when a root's side of 0 or 1 or its f32 rounding is not certain.
DVG_WN_HD int closest_quad_roots_newton(double A, double B, double C, double D, float* t32,
                                        const float* perturb = nullptr) {
    int n = 0;
    const int st = cubic_roots_certified<true>(
        A, B, C, D,
        [&](double y, float uy, double b3) -> int {
            const double t = y - b3;
            const double ut = ((double)uy + 4.5e-16 * std::fabs(y) + 9.0e-16 * std::fabs(b3)) * 1.001;
            if (!(ut < 1.0e-3)) return WIND_UNSURE;
            if (t + ut < 0.0 || t - ut > 1.0) return 0;  // not a candidate, for both
            if (!(t - ut >= 0.0 && t + ut <= 1.0)) return WIND_UNSURE;
            const float f = (float)t;
            if (!((float)(t - ut) == f && (float)(t + ut) == f)) return WIND_UNSURE;  // rounds alike
            t32[n++] = f;
            return 0;
        },
        perturb);
    return st == WIND_UNSURE ? -1 : n;
}

}  // namespace dvgb
