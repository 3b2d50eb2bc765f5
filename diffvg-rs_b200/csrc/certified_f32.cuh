// certified_f32.cuh — decisions the crate makes with f64 root solves, made in f32
// whenever margins prove the f64 computation decides the same: the winding contribution
// of a cubic segment (winding_cubic_f32) and the stroke test of a quadratic segment of
// constant radius (within_quad_f32).  Both return *_UNSURE otherwise, and the caller
// runs the f64 computation.  tests/test_winding_f32.py holds both to the oracle's f64
// decisions on random and adversarial inputs, including initial roots perturbed by the
// largest error of the fast root formulas below.
//
// Both solve a cubic t^3 + B t^2 + C t + D (normalised by its leading coefficient):
//  * the crate takes its cubic branch (leading coefficient >= 1e-6) and the normalised
//    cubic is well scaled: leading >= 1e-3 and >= max(other coefficients) / 16, so that
//    |B|, |C|, |D| <= 16, q <= 34, |r| <= 203;
//  * the number of real roots is the same in f32 and f64: |r^2 - q^3| exceeds
//    1e-3 (r^2 + |q|^3) + 1e-4 (|r| + q^2) + 1e-6, while the f32 error of r^2 - q^3 is
//    below 2.4e-5 |r| + 6e-6 q^2 (relative rounding 6e-8 on terms of at most 203 and 34);
//  * initial roots come from the trigonometric / Cardano formulas evaluated with fast
//    functions on the GPU (cos on [-pi, pi], the acos approximation of Abramowitz and
//    Stegun 4.4.45, |error| <= 7e-5, a fast power for the cube root): within ~5e-4 of the
//    exact roots given the margins above, and refined by Newton steps on the f32
//    polynomial (see each user for its convergence checks).
//
// Winding.  The crate computes the +x-ray crossings of a cubic segment in f64 (winding.rs:170-192:
// solve_cubic on the y polynomial, then x(t) > px and the sign of y'(t) at every root
// in [0, 1]).  winding_cubic_f32 decides when, in addition:
//  * every root within 0.5 of [0, 1] is refined by two Newton steps where |y'| exceeds
//    1e-2 (|a| + |b| + |c|) (after two steps the root is within ~1e-5 of the exact one,
//    as is the crate's f64 root); the last step is below 1e-4; a refined root within
//    1e-3 of 0 or 1 is undecided (the crate's t in [0, 1] test is inclusive);
//  * at a root in [0, 1], |x(t) - px| > 1e-3 (1 + |px| + max |x_k|) (the root error moves
//    x(t) by at most 6e-5 max |x_k|) and |y'(t)| > 1e-2 (|a| + |b| + |c|).
// The coefficients a, b, c, d (and those of x) are the crate's f32 expressions,
// evaluated in the same order without contraction, so both paths start from the same
// numbers.
#pragma once

#ifndef __CUDACC__
#include <cmath>
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#endif

#if defined(__CUDA_ARCH__)
#define DVG_CERT_NOINLINE __noinline__
#else
#define DVG_CERT_NOINLINE
#endif

namespace dvgb {

constexpr int WIND_UNSURE = 0x7fff;
constexpr int WITHIN_UNSURE = 2;

// acos on [-1, 1] (Abramowitz and Stegun 4.4.45: sqrt(1 - x) times a cubic in x on
// [0, 1], |error| <= 7e-5; acos(-x) = pi - acos(x)).
__host__ __device__ inline float acos_as(float x) {
    const float ax = fminf(fabsf(x), 1.0f);
    const float p = ((-0.0187293f * ax + 0.0742610f) * ax - 0.2121144f) * ax + 1.5707288f;
    const float v = sqrtf(1.0f - ax) * p;
    return x < 0.0f ? 3.14159265358979323846f - v : v;
}
__host__ __device__ inline float cos_fast(float x) {  // x in [-pi, pi]
#if defined(__CUDA_ARCH__)
    return __cosf(x);
#else
    return cosf(x);
#endif
}
__host__ __device__ inline float cbrt_fast(float x) {  // x > 0
#if defined(__CUDA_ARCH__)
    return __powf(x, 1.0f / 3.0f);
#else
    return cbrtf(x);
#endif
}

// Initial real roots of t^3 + B t^2 + C t + D into t[]; returns their number (3 or 1),
// or -1 when the discriminant is too close to zero for f32 and f64 to agree on it.
__host__ __device__ DVG_CERT_NOINLINE inline int cubic_roots_f32(float B, float C, float D, float* t) {
    const float q = (B * B - 3.0f * C) / 9.0f;
    const float r = (2.0f * B * B * B - 9.0f * B * C + 27.0f * D) / 54.0f;
    const float q3 = q * q * q, r2 = r * r;
    const float disc = r2 - q3;
    if (!(fabsf(disc) > 1.0e-3f * (r2 + fabsf(q3)) + 1.0e-4f * (fabsf(r) + q * q) + 1.0e-6f)) return -1;
    if (disc < 0.0f) {  // three real roots (q > 0 here)
        const float th = acos_as(r / sqrtf(q3));
        const float s = -2.0f * sqrtf(q);
        t[0] = s * cos_fast(th / 3.0f) - B / 3.0f;
        t[1] = s * cos_fast((th + 6.28318530717958648f) / 3.0f) - B / 3.0f;
        t[2] = s * cos_fast((th - 6.28318530717958648f) / 3.0f) - B / 3.0f;
        return 3;
    }
    const float e = sqrtf(disc);
    const float ar = r > 0.0f ? -cbrt_fast(r + e) : cbrt_fast(-r + e);
    const float br = fabsf(ar) > 1.0e-6f ? q / ar : 0.0f;
    t[0] = (ar + br) - B / 3.0f;
    return 1;
}

// The winding decision from initial roots t[0..n) of the normalised y cubic (a, b, c, d
// the crate's coefficients): Newton refinement, then the certificate described above.
__host__ __device__ inline int winding_from_roots(float a, float b, float c, float d, const float* t0, int n,
                                                  float x0, float x1, float x2, float x3, float px) {
    const float ax = -x0 + 3.0f * x1 - 3.0f * x2 + x3;
    const float bx = 3.0f * x0 - 6.0f * x1 + 3.0f * x2;
    const float cx = -3.0f * x0 + 3.0f * x1;
    const float dx = x0 - px;
    const float xm = fmaxf(fmaxf(fabsf(x0), fabsf(x1)), fmaxf(fabsf(x2), fabsf(x3)));
    const float ex = 1.0e-3f * (1.0f + fabsf(px) + xm);
    const float ed = 1.0e-2f * (fabsf(a) + fabsf(b) + fabsf(c));
    int w = 0;
    for (int i = 0; i < n; ++i) {
        float u = t0[i];
        if (!(u > -0.5f && u < 1.5f)) continue;  // far outside [0, 1]: no crossing either way
        float step = 0.0f, moved = 0.0f;
        for (int k = 0; k < 2; ++k) {  // Newton on a u^3 + b u^2 + c u + d
            const float f = ((a * u + b) * u + c) * u + d;
            const float fp = (3.0f * a * u + 2.0f * b) * u + c;
            if (!(fabsf(fp) > ed)) return WIND_UNSURE;  // a flat crossing near [0, 1]
            step = f / fp;
            u -= step;
            moved += fabsf(step);
        }
        if (!(fabsf(step) < 1.0e-4f) || !(moved < 1.0e-2f)) return WIND_UNSURE;
        if (u < -1.0e-3f || u > 1.0f + 1.0e-3f) continue;  // outside [0, 1] by the margin
        if (u <= 1.0e-3f || u >= 1.0f - 1.0e-3f) return WIND_UNSURE;
        const float tp = ((ax * u + bx) * u + cx) * u + dx;
        if (!(fabsf(tp) > ex)) return WIND_UNSURE;
        if (tp > 0.0f) {
            const float dy = (3.0f * a * u + 2.0f * b) * u + c;
            if (!(fabsf(dy) > ed)) return WIND_UNSURE;
            w += dy > 0.0f ? 1 : -1;
        }
    }
    return w;
}

__host__ __device__ inline int winding_cubic_f32(float x0, float y0, float x1, float y1, float x2, float y2, float x3,
                                                 float y3, float px, float py) {
    const float a = -y0 + 3.0f * y1 - 3.0f * y2 + y3;
    const float b = 3.0f * y0 - 6.0f * y1 + 3.0f * y2;
    const float c = -3.0f * y0 + 3.0f * y1;
    const float d = y0 - py;
    const float mcoef = fmaxf(fmaxf(fabsf(b), fabsf(c)), fabsf(d));
    if (!(fabsf(a) >= 1.0e-3f) || !(fabsf(a) * 16.0f >= mcoef)) return WIND_UNSURE;
    float t[3];
    const int n = cubic_roots_f32(b / a, c / a, d / a, t);
    if (n < 0) return WIND_UNSURE;
    return winding_from_roots(a, b, c, d, t, n, x0, x1, x2, x3, px);
}

// Stroke test of a quadratic segment with the same radius r at its three control points
// (closest.rs:20-98 with closest_point_quadratic, curve.rs:26-78): the crate keeps the
// closest of p0, p2 and the curve points at the roots in [0, 1] of the cubic
// A t^3 + B t^2 + C t + D (the derivative of the squared distance, solved in f64) and
// tests dist < r(t) (r(t) = r up to rounding).  Here: the same coefficients in f32, the
// initial roots, one Newton step, every root clamped to [0, 1] (a root just outside
// gives the end point's distance, which the crate has as a candidate anyway), and the
// smallest candidate distance d.  Decided when |d - r| > 1e-3 (1 + |p| + max |p_k| + r):
// the candidates agree with the crate's up to the root error (~1e-4 after the step) times
// |B'| (at most twice the control polygon's extent), and the distance is stationary at
// interior roots.
__host__ __device__ inline int within_quad_from_roots(const float* t0, int n, float x0, float y0, float x1, float y1,
                                                      float x2, float y2, float r, float px, float py, float A, float B,
                                                      float C, float D) {
    const float d0x = px - x0, d0y = py - y0, d2x = px - x2, d2y = py - y2;
    float d = fminf(sqrtf(d0x * d0x + d0y * d0y), sqrtf(d2x * d2x + d2y * d2y));
    for (int i = 0; i < n; ++i) {
        float u = t0[i];
        if (!(u > -0.5f && u < 1.5f)) continue;  // far outside [0, 1]: not a candidate either way
        const float fp = (3.0f * A * u + 2.0f * B) * u + C;
        if (fabsf(fp) > 0.0f) {
            const float step = (((A * u + B) * u + C) * u + D) / fp;
            if (fabsf(step) < 0.25f) u -= step;
        }
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        const float tt = 1.0f - u;
        const float w0 = tt * tt, w1 = 2.0f * tt * u, w2 = u * u;
        const float ex = (x0 * w0 + x1 * w1) + x2 * w2 - px, ey = (y0 * w0 + y1 * w1) + y2 * w2 - py;
        d = fminf(d, sqrtf(ex * ex + ey * ey));
    }
    const float pm = fmaxf(fmaxf(fmaxf(fabsf(x0), fabsf(y0)), fmaxf(fabsf(x1), fabsf(y1))),
                           fmaxf(fabsf(x2), fabsf(y2)));
    const float margin = 1.0e-3f * (1.0f + fmaxf(fabsf(px), fabsf(py)) + pm + r);
    if (d < r - margin) return 1;
    if (d > r + margin) return 0;
    return WITHIN_UNSURE;
}

__host__ __device__ DVG_CERT_NOINLINE inline int within_quad_f32(float x0, float y0, float x1, float y1, float x2,
                                                                 float y2, float r, float px, float py) {
    const float ax = x0 - 2.0f * x1 + x2, ay = y0 - 2.0f * y1 + y2;
    const float bx = -x0 + x1, by = -y0 + y1;
    const float cx = x0 - px, cy = y0 - py;
    const float A = ax * ax + ay * ay;
    const float B = 3.0f * (ax * bx + ay * by);
    const float C = 2.0f * (bx * bx + by * by) + (ax * cx + ay * cy);
    const float D = bx * cx + by * cy;
    const float mcoef = fmaxf(fmaxf(fabsf(B), fabsf(C)), fabsf(D));
    if (!(A >= 1.0e-3f) || !(A * 16.0f >= mcoef)) return WITHIN_UNSURE;
    float t[3];
    const int n = cubic_roots_f32(B / A, C / A, D / A, t);
    if (n < 0) return WITHIN_UNSURE;
    return within_quad_from_roots(t, n, x0, y0, x1, y1, x2, y2, r, px, py, A, B, C, D);
}

}  // namespace dvgb
