// device.cuh — device-side scene evaluation for the diffvg hot path (sm_100a).
//
// Per-sample evaluation with the crate's CPU semantics (src/backward/sampling.rs,
// src/distance/*.rs): stroke "within distance" and fill winding-number tests,
// evaluated over the crate's median-split BVHs (rebuilt on the host with the same
// topology, walked here with skip links).  Arithmetic mirrors the crate: f32
// everywhere, f64 exactly where the crate casts to f64 (root solves), and the
// translation unit is compiled with -fmad=false so that no multiply-add is fused
// (Rust never fuses), which keeps inside/outside decisions bit-identical.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "prepare.hpp"  // ShapeFlags shared with the host preparation
// Set by a translation unit before including this header: DVG_EXACT_ROOT_SOLVES, the cubic
// winding runs the crate's root formula; DVG_EXACT_CLOSEST_QUAD, the quadratic closest
// point does (both also without them whenever the certified shortcut is not sure).
#ifndef DVG_EXACT_ROOT_SOLVES
#define DVG_EXACT_ROOT_SOLVES 0
#endif
#ifndef DVG_EXACT_CLOSEST_QUAD
#define DVG_EXACT_CLOSEST_QUAD DVG_EXACT_ROOT_SOLVES
#endif
#include "winding_newton.cuh"

namespace dvgb {

constexpr int TILE = 16;          // tile edge in pixels (the crate's TILE_SIZE)
constexpr int TILE_PIXELS = TILE * TILE;
constexpr float PI_F = 3.14159265358979323846f;
constexpr float HALF_PI_F = 1.57079632679489661923f;

enum : int { K_CIRCLE = 0, K_RECT = 1, K_PATH = 2, K_ELLIPSE = 3 };
enum : int { P_NONE = 0, P_SOLID = 1, P_LINEAR = 2, P_RADIAL = 3 };
enum : int { F_BOX = 0, F_TENT = 1, F_PARABOLIC = 2, F_HANN = 3, F_GAUSSIAN = 4 };
enum : int { PF_CLOSED = 1, PF_APPROX = 2, PF_THICK = 4, PF_STYLED = 8, PF_JOIN_SHIFT = 4, PF_CAP_SHIFT = 6 };
enum : int { JOIN_MITER = 0, JOIN_BEVEL = 1, JOIN_ROUND = 2, CAP_BUTT = 0, CAP_SQUARE = 1, CAP_ROUND = 2 };

// Device status bits written by kernels (never a trap: the host reads them).
enum : unsigned { ST_FRAGMENT_OVERFLOW = 1u, ST_BVH_LIMIT = 2u, ST_REFIT_LAYOUT = 4u };

struct DevScene {
    int width, height;
    int num_groups, num_shapes, num_paints, num_paths;
    int styled;  // some path strokes with non-round joins or caps
    int filter_type;
    float filter_radius;
    int filter_ri;
    float bg[4];
    const float* bg_image;
    // groups
    const float* g_c2s;  // 9 per group (full canvas_to_shape)
    const float* g_s2c;  // 9 per group
    const int4* g_info;  // fill paint, stroke paint, fill rule, 0
    const int4* g_bvh;   // node off, node count, list off, list count
    const int* g_shape_list;
    const float4* gn_bounds;
    const int4* gn_meta;  // skip, leaf start, count, right child (left child = node + 1)
    const int* gl_shapes;
    // shapes
    const int4* s_info;  // kind, flags, path index, 0
    const float4* s_params;
    const float* s_inv;    // 6 per shape
    const float* s_xform;  // 9 per shape
    const float* s_stroke;
    const float4* s_box;     // padded group-space bounds (scene re-preparation only)
    const float* s_padmul;   // stroke-pad multiplier (scene re-preparation only)
    // paths
    const int4* p_info;  // 2 per path: (seg off, seg cnt, node off, node cnt), (pt off, pt cnt, ctrl off, flags)
    const int* p_shape;  // shape id per path
    const float* p_miter;  // miter limit (>= 1) per path
    const float4* pn_bounds;
    const int4* pn_meta;
    const int* pl_segs;
    const float4* seg_p;  // 2 per segment
    const float4* seg_r;
    const int4* seg_meta;  // kind, segment index, point id, shape
    const float2* points;
    const float* thickness;
    const uint8_t* ncp;
    // paints
    const int4* paint_info;  // kind, stop off, stop count, 0
    const float4* paint_params;
    const float* stop_offsets;
    const float4* stop_colors;
    // boundary tables
    int boundary_ok;
    int bcdf_n;
    const float* shape_len;
    const float* bcdf;
    const float* bpmf;
    const int* b_shape;
    const int* b_group;
    const int4* path_cdf_info;
    const float* path_cdf;
    const float* path_pmf;
    const int* path_pid;
    const float* path_len;
    const float4* g_bbox;  // conservative canvas-space group boxes (binning, distance search skips)
    // tile binning
    int tiles_x, tiles_y;
    const int* tile_offsets;
    const int* tile_entries;
};

// ------------------------------------------------------------------ small math
__device__ __forceinline__ float clampf(float v, float lo, float hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}
__device__ __forceinline__ float len2(float x, float y) { return sqrtf(x * x + y * y); }
// Rust `f as i32` (saturating, NaN -> 0) — cvt.rzi.s32.f32 has exactly these semantics.
__device__ __forceinline__ int f2i(float f) { return __float2int_rz(f); }
__device__ __forceinline__ float2 xf6(const float* m, float2 p) {  // Mat3::transform_point
    return make_float2(m[0] * p.x + m[1] * p.y + m[2], m[3] * p.x + m[4] * p.y + m[5]);
}
__device__ __forceinline__ float2 xf9(const float* m, float2 p) {
    return make_float2(m[0] * p.x + m[1] * p.y + m[2], m[3] * p.x + m[4] * p.y + m[5]);
}
// distance/utils.rs:7-16: identity shortcut, singular -> unchanged
__device__ __forceinline__ float2 shape_local_dist(const DevScene& S, int s, float2 p) {
    int flags = S.s_info[s].y;
    if (flags & SF_IDENTITY) return p;
    if (flags & SF_INVERTIBLE) return xf6(S.s_inv + 6 * s, p);
    return p;
}
// backward/math.rs:131-135: no identity shortcut, singular -> identity
__device__ __forceinline__ float2 shape_local_bwd(const DevScene& S, int s, float2 p) {
    if (S.s_info[s].y & SF_INVERTIBLE) return xf6(S.s_inv + 6 * s, p);
    return p;
}

// ------------------------------------------------------------------ polynomial roots (f64, distance/utils.rs:48-123)
// Out-of-line wrappers: one copy of each libm body per kernel instead of one per call site.
static __device__ __noinline__ double dvg_acos(double x) { return acos(x); }
static __device__ __noinline__ double dvg_cos(double x) { return cos(x); }
static __device__ __noinline__ double dvg_pow(double x, double y) { return pow(x, y); }
static __device__ __noinline__ float dvg_sinf(float x) { return sinf(x); }
static __device__ __noinline__ float dvg_cosf(float x) { return cosf(x); }
static __device__ __noinline__ float dvg_expf(float x) { return expf(x); }
static __device__ __noinline__ float dvg_atan2f(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ bool solve_quadratic(double a, double b, double c, double t[2]) {
    const double eps = 1.0e-12;
    if (fabs(a) < eps) {
        if (fabs(b) < eps) return false;
        double root = -c / b;
        t[0] = root;
        t[1] = root;
        return true;
    }
    double discrim = b * b - 4.0 * a * c;
    if (discrim < 0.0) return false;
    double root = sqrt(discrim);
    if (fabs(root) < eps) {
        double r = -0.5 * b / a;
        t[0] = r;
        t[1] = r;
        return true;
    }
    double q = (b < 0.0) ? -0.5 * (b - root) : -0.5 * (b + root);
    if (fabs(q) < eps) {
        double inv = 0.5 / a;
        t[0] = (-b - root) * inv;
        t[1] = (-b + root) * inv;
    } else {
        t[0] = q / a;
        t[1] = c / q;
    }
    if (t[0] > t[1]) {
        double tmp = t[0];
        t[0] = t[1];
        t[1] = tmp;
    }
    return true;
}
__device__ __forceinline__ double cbrt_pow(double x) {
    if (x > 0.0) return dvg_pow(x, 1.0 / 3.0);
    if (x < 0.0) return -dvg_pow(-x, 1.0 / 3.0);
    return 0.0;
}
static __device__ __noinline__ int solve_cubic(double a, double b, double c, double d, double t[3]) {
    if (fabs(a) < 1.0e-6) {
        double r2[2];
        if (solve_quadratic(b, c, d, r2)) {
            t[0] = r2[0];
            t[1] = r2[1];
            return 2;
        }
        return 0;
    }
    b = b / a;
    c = c / a;
    d = d / a;
    double q = (b * b - 3.0 * c) / 9.0;
    double r = (2.0 * b * b * b - 9.0 * b * c + 27.0 * d) / 54.0;
    const double TWO_PI = 6.283185307179586476925286766559;
    if (r * r < q * q * q) {
        double theta = dvg_acos(r / sqrt(q * q * q));
        double sq = sqrt(q);
        t[0] = -2.0 * sq * dvg_cos(theta / 3.0) - b / 3.0;
        t[1] = -2.0 * sq * dvg_cos((theta + TWO_PI) / 3.0) - b / 3.0;
        t[2] = -2.0 * sq * dvg_cos((theta - TWO_PI) / 3.0) - b / 3.0;
        return 3;
    }
    double ar = (r > 0.0) ? -cbrt_pow(r + sqrt(r * r - q * q * q)) : cbrt_pow(-r + sqrt(r * r - q * q * q));
    double br = (fabs(ar) > 1.0e-6) ? q / ar : 0.0;
    t[0] = (ar + br) - b / 3.0;
    return 1;
}

// ------------------------------------------------------------------ closest points (distance/curve.rs)
struct CPRes {
    float cx, cy, t, dist;
};
__device__ __forceinline__ CPRes closest_line(float2 p, float ax, float ay, float bx, float by) {  // curve.rs:10-21
    float abx = bx - ax, aby = by - ay;
    float denom = abx * abx + aby * aby;
    if (denom <= 1.0e-10f) return CPRes{ax, ay, 0.0f, len2(p.x - ax, p.y - ay)};
    float t = clampf(((p.x - ax) * abx + (p.y - ay) * aby) / denom, 0.0f, 1.0f);
    float cx = ax + abx * t, cy = ay + aby * t;
    return CPRes{cx, cy, t, len2(p.x - cx, p.y - cy)};
}
static __device__ __noinline__ CPRes closest_quad_approx_v(float2 pt, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7);
__device__ __forceinline__ CPRes closest_quad_approx(float2 pt, const float* q) {
    return closest_quad_approx_v(pt, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]);
}
static __device__ __noinline__ CPRes closest_quad_approx_v(float2 pt, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7) {
    const float q[8] = {a0, a1, a2, a3, a4, a5, a6, a7};  // curve.rs:267-296
    float b0x = q[0] - pt.x, b0y = q[1] - pt.y, b1x = q[2] - pt.x, b1y = q[3] - pt.y;
    float b2x = q[4] - pt.x, b2y = q[5] - pt.y;
    float a = b0x * b2y - b0y * b2x;
    float b = 2.0f * (b1x * b0y - b1y * b0x);
    float d = 2.0f * (b2x * b1y - b2y * b1x);
    float f = b * d - a * a;
    float d21x = b2x - b1x, d21y = b2y - b1y, d10x = b1x - b0x, d10y = b1y - b0y, d20x = b2x - b0x, d20y = b2y - b0y;
    float gx = (d21x * b) + (d10x * d) + (d20x * a);
    float gy = (d21y * b) + (d10y * d) + (d20y * a);
    gx = gx * 2.0f;
    gy = gy * 2.0f;
    float gfx = gy, gfy = -gx;
    float t = 0.0f;
    float denom = gfx * gfx + gfy * gfy;
    if (denom > 1.0e-8f) {
        float s = -f / denom;
        float ppx = gfx * s, ppy = gfy * s;
        float d0px = b0x - ppx, d0py = b0y - ppy;
        float ap = d0px * d20y - d0py * d20x;
        float bp = 2.0f * (d10x * d0py - d10y * d0px);
        float denom2 = 2.0f * a + b + d;
        if (fabsf(denom2) > 1.0e-8f) t = clampf((ap + bp) / denom2, 0.0f, 1.0f);
    }
    float tt = 1.0f - t;
    float w0 = tt * tt, w1 = 2.0f * tt * t, w2 = t * t;
    float cx = q[0] * w0 + q[2] * w1 + q[4] * w2, cy = q[1] * w0 + q[3] * w1 + q[5] * w2;
    return CPRes{cx, cy, t, len2(pt.x - cx, pt.y - cy)};
}
// The crate's candidates: its f64 roots (solve_cubic) in [0, 1], as f32 parameters (inline
// where it is the only path, as for the winding).
#if DVG_EXACT_CLOSEST_QUAD
#define DVG_QUAD_EXACT_ATTR __forceinline__
#else
#define DVG_QUAD_EXACT_ATTR __noinline__
#endif
static __device__ DVG_QUAD_EXACT_ATTR int closest_quad_candidates_exact(double A, double B, double C, double D,
                                                                        float* t32) {
    double r[3];
    const int nr = solve_cubic(A, B, C, D, r);
    int n = 0;
    for (int i = 0; i < nr; ++i)
        if (r[i] >= 0.0 && r[i] <= 1.0) t32[n++] = (float)r[i];
    return n;
}
static __device__ __noinline__ CPRes closest_quad_v(float2 pt, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7, bool approx);
__device__ __forceinline__ CPRes closest_quad(float2 pt, const float* q, bool approx) {
    return closest_quad_v(pt, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], approx);
}
static __device__ __noinline__ CPRes closest_quad_v(float2 pt, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7, bool approx) {
    const float q[8] = {a0, a1, a2, a3, a4, a5, a6, a7};  // curve.rs:26-78
    if (approx) return closest_quad_approx(pt, q);
    float best_t = 0.0f, bx = q[0], by = q[1];
    float best = len2(pt.x - q[0], pt.y - q[1]);
    float de = len2(pt.x - q[4], pt.y - q[5]);
    if (de < best) {
        best = de;
        bx = q[4];
        by = q[5];
        best_t = 1.0f;
    }
    double ax = (double)(q[0] - 2.0f * q[2] + q[4]);
    double ay = (double)(q[1] - 2.0f * q[3] + q[5]);
    double bbx = (double)(-q[0] + q[2]);
    double bby = (double)(-q[1] + q[3]);
    double cx = (double)(q[0] - pt.x);
    double cy = (double)(q[1] - pt.y);
    double A = ax * ax + ay * ay;
    double B = 3.0 * (ax * bbx + ay * bby);
    double Cc = 2.0 * (bbx * bbx + bby * bby) + (ax * cx + ay * cy);
    double D = bbx * cx + bby * cy;
    // the crate's candidates t32 = (float)t of the roots in [0, 1]: certified without its
    // acos / cos / pow when their side of 0 and 1 and their f32 rounding provably agree
    float cand[3];
#if DVG_EXACT_CLOSEST_QUAD
    const int n = closest_quad_candidates_exact(A, B, Cc, D, cand);
#else
    int n = closest_quad_roots_newton(A, B, Cc, D, cand);
    if (n < 0) n = closest_quad_candidates_exact(A, B, Cc, D, cand);
#endif
    for (int i = 0; i < n; ++i) {
        float t32 = cand[i];
        float tt = 1.0f - t32;
        float w0 = tt * tt, w1 = 2.0f * tt * t32, w2 = t32 * t32;
        float px = (q[0] * w0 + q[2] * w1) + q[4] * w2;
        float py = (q[1] * w0 + q[3] * w1) + q[5] * w2;
        float dist = len2(pt.x - px, pt.y - py);
        if (dist < best) {
            best = dist;
            bx = px;
            by = py;
            best_t = t32;
        }
    }
    return CPRes{bx, by, best_t, best};
}
static __device__ __noinline__ CPRes closest_cubic_approx_v(float2 pt, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7);
__device__ __forceinline__ CPRes closest_cubic_approx(float2 pt, const float* q) {
    return closest_cubic_approx_v(pt, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]);
}
static __device__ __noinline__ CPRes closest_cubic_approx_v(float2 pt, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7) {
    const float q[8] = {a0, a1, a2, a3, a4, a5, a6, a7};  // curve.rs:81-119
    float inv = 1.0f / 8.0f;
    float prevx = q[0], prevy = q[1], prev_t = 0.0f;
    float bx = q[0], by = q[1], best_t = 0.0f, best = len2(pt.x - q[0], pt.y - q[1]);
    for (int i = 1; i <= 8; ++i) {
        float t = (float)i * inv;
        float tt = 1.0f - t;
        float tt2 = tt * tt, t2 = t * t;
        float a = tt2 * tt, b = 3.0f * tt2 * t, c = 3.0f * tt * t2, d = t2 * t;
        float cxx = a * q[0] + b * q[2] + c * q[4] + d * q[6];
        float cyy = a * q[1] + b * q[3] + c * q[5] + d * q[7];
        CPRes r = closest_line(pt, prevx, prevy, cxx, cyy);
        float lt = prev_t + r.t * (t - prev_t);
        if (r.dist < best) {
            best = r.dist;
            bx = r.cx;
            by = r.cy;
            best_t = lt;
        }
        prevx = cxx;
        prevy = cyy;
        prev_t = t;
    }
    return CPRes{bx, by, best_t, best};
}
static __device__ __noinline__ CPRes closest_cubic_v(float2 pt, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7, bool approx);
__device__ __forceinline__ CPRes closest_cubic(float2 pt, const float* q, bool approx) {
    return closest_cubic_v(pt, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], approx);
}
static __device__ __noinline__ CPRes closest_cubic_v(float2 pt, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7, bool approx) {
    const float q[8] = {a0, a1, a2, a3, a4, a5, a6, a7};  // curve.rs:124-264
    if (approx) return closest_cubic_approx(pt, q);
    float best_t = 0.0f, bx = q[0], by = q[1];
    float best = len2(pt.x - q[0], pt.y - q[1]);
    float de = len2(pt.x - q[6], pt.y - q[7]);
    if (de < best) {
        best = de;
        bx = q[6];
        by = q[7];
        best_t = 1.0f;
    }
    double ax = (double)(-q[0] + 3.0f * q[2] - 3.0f * q[4] + q[6]);
    double ay = (double)(-q[1] + 3.0f * q[3] - 3.0f * q[5] + q[7]);
    double bxx = (double)(3.0f * q[0] - 6.0f * q[2] + 3.0f * q[4]);
    double byy = (double)(3.0f * q[1] - 6.0f * q[3] + 3.0f * q[5]);
    double cx = (double)(-3.0f * q[0] + 3.0f * q[2]);
    double cy = (double)(-3.0f * q[1] + 3.0f * q[3]);
    double dx = (double)(q[0] - pt.x);
    double dy = (double)(q[1] - pt.y);
    double a = 3.0 * (ax * ax + ay * ay);
    if (fabs(a) < 1.0e-10) return CPRes{bx, by, best_t, best};
    double b = 5.0 * (ax * bxx + ay * byy);
    double c = 4.0 * (ax * cx + ay * cy) + 2.0 * (bxx * bxx + byy * byy);
    double d = 3.0 * ((bxx * cx + byy * cy) + (ax * dx + ay * dy));
    double e = (cx * cx + cy * cy) + 2.0 * (dx * bxx + dy * byy);
    double f = dx * cx + dy * cy;
    b = b / a;
    c = c / a;
    d = d / a;
    e = e / a;
    f = f / a;
    double p1a = (2.0 / 5.0) * c - (4.0 / 25.0) * b * b;
    double p1b = (3.0 / 5.0) * d - (3.0 / 25.0) * b * c;
    double p1c = (4.0 / 5.0) * e - (2.0 / 25.0) * b * d;
    double p1d = f - b * e / 25.0;
    double q_root = -b / 5.0;
    double pr[3];
    int num_p = solve_cubic(p1a, p1b, p1c, p1d, pr);
    double iv[4];
    int ni = 0;
    if (q_root >= 0.0 && q_root <= 1.0) iv[ni++] = q_root;
    for (int i = 0; i < num_p; ++i) iv[ni++] = pr[i];
    for (int j = 1; j < ni; ++j) {
        int k = j;
        while (k > 0 && iv[k - 1] > iv[k]) {
            double tmp = iv[k - 1];
            iv[k - 1] = iv[k];
            iv[k] = tmp;
            k -= 1;
        }
    }
    double lower = 0.0;
    for (int j = 0; j <= ni; ++j) {
        if (j < ni && iv[j] < 0.0) continue;
        double upper = (j < ni) ? fmin(iv[j], 1.0) : 1.0;
        double lb = lower, ub = upper;
        double lbe = ((((lb + b) * lb + c) * lb + d) * lb + e) * lb + f;
        double ube = ((((ub + b) * ub + c) * ub + d) * ub + e) * ub + f;
        if (lbe * ube > 0.0) {
            lower = upper;
            continue;
        }
        if (lbe > ube) {
            double t0 = lb;
            lb = ub;
            ub = t0;
        }
        double t = 0.5 * (lb + ub);
        for (int it = 0; it < 20; ++it) {
            if (!(t >= lb && t <= ub)) t = 0.5 * (lb + ub);
            double v = ((((t + b) * t + c) * t + d) * t + e) * t + f;
            if (fabs(v) < 1.0e-5 || it == 19) break;
            if (v > 0.0)
                ub = t;
            else
                lb = t;
            double dv = (((5.0 * t + 4.0 * b) * t + 3.0 * c) * t + 2.0 * d) * t + e;
            t -= v / dv;
        }
        if (t >= 0.0 && t <= 1.0) {
            float t32 = (float)t;
            float tt = 1.0f - t32;
            float w0 = tt * tt * tt, w1 = 3.0f * tt * tt * t32, w2 = 3.0f * tt * t32 * t32, w3 = t32 * t32 * t32;
            float px = ((q[0] * w0 + q[2] * w1) + q[4] * w2) + q[6] * w3;
            float py = ((q[1] * w0 + q[3] * w1) + q[5] * w2) + q[7] * w3;
            float dist = len2(pt.x - px, pt.y - py);
            if (dist < best) {
                best = dist;
                bx = px;
                by = py;
                best_t = t32;
            }
        }
        if (upper >= 1.0) break;
        lower = upper;
    }
    return CPRes{bx, by, best_t, best};
}

// ------------------------------------------------------------------ segments
struct SegGeom {
    float q[8];
    float r[4];
    int kind;
};
__device__ __forceinline__ void load_seg(const DevScene& S, int sidx, SegGeom& sg) {
    float4 a = __ldg(&S.seg_p[2 * sidx]);
    float4 b = __ldg(&S.seg_p[2 * sidx + 1]);
    float4 r = __ldg(&S.seg_r[sidx]);
    sg.q[0] = a.x; sg.q[1] = a.y; sg.q[2] = a.z; sg.q[3] = a.w;
    sg.q[4] = b.x; sg.q[5] = b.y; sg.q[6] = b.z; sg.q[7] = b.w;
    sg.r[0] = r.x; sg.r[1] = r.y; sg.r[2] = r.z; sg.r[3] = r.w;
    sg.kind = __ldg(&S.seg_meta[sidx].x);
}
__device__ __forceinline__ CPRes seg_closest(const SegGeom& sg, float2 p, bool approx) {
    if (sg.kind == 0) return closest_line(p, sg.q[0], sg.q[1], sg.q[2], sg.q[3]);
    if (sg.kind == 1) return closest_quad(p, sg.q, approx);
    return closest_cubic(p, sg.q, approx);
}
__device__ __forceinline__ float seg_radius(const SegGeom& s, float t) {  // closest.rs:66-79
    if (s.kind == 0) return s.r[0] + t * (s.r[1] - s.r[0]);
    float tt = 1.0f - t;
    if (s.kind == 1) return tt * tt * s.r[0] + 2.0f * tt * t * s.r[1] + t * t * s.r[2];
    return tt * tt * tt * s.r[0] + 3.0f * tt * tt * t * s.r[1] + 3.0f * tt * t * t * s.r[2] + t * t * t * s.r[3];
}
// The crate's cubic crossings: its f64 roots (solve_cubic) and decisions (winding.rs:170-192).
// Out of line where it is the certified path's fallback (rarely run), inline where it is
// the only path.
#if DVG_EXACT_ROOT_SOLVES
#define DVG_WIND_EXACT_ATTR __forceinline__
#else
#define DVG_WIND_EXACT_ATTR __noinline__
#endif
static __device__ DVG_WIND_EXACT_ATTR int winding_cubic_exact(double a, double b, double c, double d, double ax,
                                                              double bx, double cx, double dx) {
    double r[3];
    int nr = solve_cubic(a, b, c, d, r);
    int w = 0;
    for (int i = 0; i < nr; ++i) {
        double t = r[i];
        if (t >= 0.0 && t <= 1.0) {
            double tp = ax * t * t * t + bx * t * t + cx * t + dx;
            if (tp > 0.0) w += (3.0 * a * t * t + 2.0 * b * t + c) > 0.0 ? 1 : -1;
        }
    }
    return w;
}
// winding.rs:118-192
static __device__ __noinline__ int winding_segment_v(int kind, float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7, float2 pt) {
    const float q[8] = {a0, a1, a2, a3, a4, a5, a6, a7};
    if (kind == 0) {
        float dy = q[3] - q[1];
        if (fabsf(dy) <= 1.0e-8f) return 0;
        float t = (pt.y - q[1]) / dy;
        if (t >= 0.0f && t <= 1.0f) {
            float tp = q[0] - pt.x + t * (q[2] - q[0]);
            if (tp >= 0.0f) return dy > 0.0f ? 1 : -1;
        }
        return 0;
    }
    if (kind == 1) {
        double a = (double)(q[1] - 2.0f * q[3] + q[5]);
        double b = (double)(-2.0f * q[1] + 2.0f * q[3]);
        double c = (double)(q[1] - pt.y);
        double r[2];
        int nr = 0;
        if (fabs(a) < 1.0e-12) {
            if (fabs(b) > 1.0e-12) {
                r[0] = -c / b;
                nr = 1;
            }
        } else if (solve_quadratic(a, b, c, r)) {
            nr = 2;
        }
        double ax = (double)(q[0] - 2.0f * q[2] + q[4]);
        double bx = (double)(-2.0f * q[0] + 2.0f * q[2]);
        double cx = (double)(q[0] - pt.x);
        int w = 0;
        for (int i = 0; i < nr; ++i) {
            double t = r[i];
            if (t >= 0.0 && t <= 1.0) {
                double tp = ax * t * t + bx * t + cx;
                if (tp > 0.0) w += (2.0 * a * t + b) > 0.0 ? 1 : -1;
            }
        }
        return w;
    }
    double a = (double)(-q[1] + 3.0f * q[3] - 3.0f * q[5] + q[7]);
    double b = (double)(3.0f * q[1] - 6.0f * q[3] + 3.0f * q[5]);
    double c = (double)(-3.0f * q[1] + 3.0f * q[3]);
    double d = (double)(q[1] - pt.y);
    double ax = (double)(-q[0] + 3.0f * q[2] - 3.0f * q[4] + q[6]);
    double bx = (double)(3.0f * q[0] - 6.0f * q[2] + 3.0f * q[4]);
    double cx = (double)(-3.0f * q[0] + 3.0f * q[2]);
    double dx = (double)(q[0] - pt.x);
#if DVG_EXACT_ROOT_SOLVES
    return winding_cubic_exact(a, b, c, d, ax, bx, cx, dx);
#else
    // the crate's decisions without its f64 acos / cos / pow whenever they provably agree
    const int wn = winding_cubic_newton(a, b, c, d, ax, bx, cx, dx);
    return wn != WIND_UNSURE ? wn : winding_cubic_exact(a, b, c, d, ax, bx, cx, dx);
#endif
}
__device__ __forceinline__ int winding_segment(const SegGeom& s, float2 pt) {
    return winding_segment_v(s.kind, s.q[0], s.q[1], s.q[2], s.q[3], s.q[4], s.q[5], s.q[6], s.q[7], pt);
}

// ------------------------------------------------------------------ exact-result culling
// A segment whose control-point hull lies strictly beyond the +x ray by more than
// the rounding of the crate's root solve cannot add a crossing: the computed
// polynomial then has no root in [0,1] with x(t) > pt.x, so winding_segment would
// return 0.  The margin is ~300x the worst-case f32 coefficient error
// (~3e-6 * max |coordinate|), so skipping such segments never changes a result.
__device__ __forceinline__ float cull_margin(const SegGeom& s, float2 p) {
    float m = fmaxf(fabsf(p.x), fabsf(p.y));
#pragma unroll
    for (int k = 0; k < 8; ++k) m = fmaxf(m, fabsf(s.q[k]));
    return 1.0e-3f * (1.0f + m);
}
__device__ __forceinline__ bool ray_misses_segment(const SegGeom& s, float2 p) {
    float ymin = fminf(fminf(s.q[1], s.q[3]), fminf(s.q[5], s.q[7]));
    float ymax = fmaxf(fmaxf(s.q[1], s.q[3]), fmaxf(s.q[5], s.q[7]));
    float xmax = fmaxf(fmaxf(s.q[0], s.q[2]), fmaxf(s.q[4], s.q[6]));
    float m = cull_margin(s, p);
    return p.y < ymin - m || p.y > ymax + m || p.x > xmax + m;
}
// A point farther than max radius (+margin) outside the control-point box of a
// segment cannot satisfy dist < radius(t): the closest point lies in the hull.
__device__ __forceinline__ bool stroke_misses_segment(const SegGeom& s, float2 p) {
    float xmin = fminf(fminf(s.q[0], s.q[2]), fminf(s.q[4], s.q[6]));
    float xmax = fmaxf(fmaxf(s.q[0], s.q[2]), fmaxf(s.q[4], s.q[6]));
    float ymin = fminf(fminf(s.q[1], s.q[3]), fminf(s.q[5], s.q[7]));
    float ymax = fmaxf(fmaxf(s.q[1], s.q[3]), fmaxf(s.q[5], s.q[7]));
    float r = fmaxf(fmaxf(s.r[0], s.r[1]), fmaxf(s.r[2], s.r[3]));
    float m = cull_margin(s, p) + 1.0e-5f * fabsf(r);
    r = r + m;
    return p.x < xmin - r || p.x > xmax + r || p.y < ymin - r || p.y > ymax + r;
}

// Lower bound on the distance from p to a cubic segment, for rejecting stroke
// tests before the exact closest-point solve.  The 16-chord polyline through
// B(k/16) lies within e = (h^2/8) max|B''| = (3 / (4 * 16^2)) max(|q0-2q1+q2|,
// |q1-2q2+q3|) of the curve (linear-interpolation error, |B''| <= 6 max|second
// difference|), so dist(p, curve) >= dist(p, polyline) - e.  Whenever this bound
// exceeds the segment's largest radius by the culling margin (far above the f32
// rounding of the polyline and of the crate's closest point), the crate's
// `dist < radius(t)` test is false, so skipping the solve never changes a result.
static __device__ __noinline__ float cubic_dist_lower(float px, float py, float a0, float a1, float a2, float a3,
                                                     float a4, float a5, float a6, float a7) {
    const float ax = -a0 + 3.0f * a2 - 3.0f * a4 + a6, ay = -a1 + 3.0f * a3 - 3.0f * a5 + a7;
    const float bx = 3.0f * a0 - 6.0f * a2 + 3.0f * a4, by = 3.0f * a1 - 6.0f * a3 + 3.0f * a5;
    const float cx = -3.0f * a0 + 3.0f * a2, cy = -3.0f * a1 + 3.0f * a3;
    float best = INFINITY;  // squared distance to the polyline
    float vx = a0 - px, vy = a1 - py;
#pragma unroll 4
    for (int k = 1; k <= 16; ++k) {
        const float t = (float)k * (1.0f / 16.0f);
        const float wx = (k == 16 ? a6 : ((ax * t + bx) * t + cx) * t + a0) - px;
        const float wy = (k == 16 ? a7 : ((ay * t + by) * t + cy) * t + a1) - py;
        const float ex = wx - vx, ey = wy - vy;
        const float ee = ex * ex + ey * ey, de = -(vx * ex + vy * ey);
        float d2;
        if (de <= 0.0f || ee <= 0.0f) d2 = vx * vx + vy * vy;
        else if (de >= ee) d2 = wx * wx + wy * wy;
        else d2 = fmaxf(vx * vx + vy * vy - de * (de / ee), 0.0f);
        best = fminf(best, d2);
        vx = wx;
        vy = wy;
    }
    const float s0x = a0 - 2.0f * a2 + a4, s0y = a1 - 2.0f * a3 + a5;
    const float s1x = a2 - 2.0f * a4 + a6, s1y = a3 - 2.0f * a5 + a7;
    const float e = (3.0f / 1024.0f) * sqrtf(fmaxf(s0x * s0x + s0y * s0y, s1x * s1x + s1y * s1y));
    return sqrtf(best) - e;
}
__device__ __forceinline__ bool stroke_far_from_cubic(const SegGeom& s, float2 p) {
    float r = fmaxf(fmaxf(s.r[0], s.r[1]), fmaxf(s.r[2], s.r[3]));
    float m = cull_margin(s, p) + 1.0e-5f * fabsf(r);
    return cubic_dist_lower(p.x, p.y, s.q[0], s.q[1], s.q[2], s.q[3], s.q[4], s.q[5], s.q[6], s.q[7]) > r + m;
}

// ------------------------------------------------------------------ stroke joins and caps
// An extension: the crate strokes every path with round joins and caps (its join /
// cap fields only pad bounds, src/renderer/prepare.rs:207-210).  A path flagged
// PF_STYLED strokes its segment bodies as the crate does, except at vertices whose
// join or cap is not round: there a closest point exactly at the segment's end does
// not count, and the join or cap region is added instead.  Bevel: the triangle
// between the vertex and the two outer offset points; miter: the quad through the
// offset lines' intersection while that lies within miter-limit radii of the vertex
// (else bevel); butt: nothing; square: a rectangle one radius long and two wide
// beyond the end.  Regions are closed sets, so they meet the bodies without cracks.
__device__ __forceinline__ bool end_excluded(int pflags, int seg, int nseg, float t) {
    const bool at0 = t == 0.0f, at1 = t == 1.0f;
    if (!(pflags & PF_STYLED) || !(at0 || at1)) return false;
    const bool join = (pflags & PF_CLOSED) || (at0 ? seg > 0 : seg < nseg - 1);
    if (join) return ((pflags >> PF_JOIN_SHIFT) & 3) != JOIN_ROUND;
    return ((pflags >> PF_CAP_SHIFT) & 3) != CAP_ROUND;
}
// Tangent directions at t = 0 and t = 1 from the control points (degenerate legs
// skipped; lines and quadratics repeat their last point).
__device__ __forceinline__ float2 seg_dir0(float4 a, float4 b) {
    float2 d = make_float2(a.z - a.x, a.w - a.y);
    if (d.x == 0.0f && d.y == 0.0f) d = make_float2(b.x - a.x, b.y - a.y);
    if (d.x == 0.0f && d.y == 0.0f) d = make_float2(b.z - a.x, b.w - a.y);
    return d;
}
__device__ __forceinline__ float2 seg_dir1(float4 a, float4 b) {
    float2 d = make_float2(b.z - b.x, b.w - b.y);
    if (d.x == 0.0f && d.y == 0.0f) d = make_float2(b.z - a.z, b.w - a.w);
    if (d.x == 0.0f && d.y == 0.0f) d = make_float2(b.z - a.x, b.w - a.y);
    return d;
}
__device__ __forceinline__ float cross2f(float ax, float ay, float bx, float by) { return ax * by - ay * bx; }
__device__ __forceinline__ bool in_triangle(float2 p, float2 a, float2 b, float2 c) {
    const float d1 = cross2f(b.x - a.x, b.y - a.y, p.x - a.x, p.y - a.y);
    const float d2 = cross2f(c.x - b.x, c.y - b.y, p.x - b.x, p.y - b.y);
    const float d3 = cross2f(a.x - c.x, a.y - c.y, p.x - c.x, p.y - c.y);
    const bool neg = d1 < 0.0f || d2 < 0.0f || d3 < 0.0f, pos = d1 > 0.0f || d2 > 0.0f || d3 > 0.0f;
    return !(neg && pos);
}
__device__ __forceinline__ bool join_hit(float2 p, float2 v, float2 din, float2 dout, float r, int join, float limit) {
    const float li = sqrtf(din.x * din.x + din.y * din.y), lo = sqrtf(dout.x * dout.x + dout.y * dout.y);
    if (!(li > 0.0f) || !(lo > 0.0f) || !(r > 0.0f)) return false;
    din = make_float2(din.x / li, din.y / li);
    dout = make_float2(dout.x / lo, dout.y / lo);
    const float cr = cross2f(din.x, din.y, dout.x, dout.y);
    if (fabsf(cr) < 1.0e-6f) return false;  // straight on (no gap) or a reversal (no outer side)
    const float sg = cr > 0.0f ? 1.0f : -1.0f;  // the outer side is right of travel on a left turn
    const float2 a = make_float2(v.x + r * sg * din.y, v.y - r * sg * din.x);
    const float2 b = make_float2(v.x + r * sg * dout.y, v.y - r * sg * dout.x);
    if (join == JOIN_MITER) {
        const float s = cross2f(b.x - a.x, b.y - a.y, dout.x, dout.y) / cr;
        const float2 m = make_float2(a.x + s * din.x, a.y + s * din.y);
        const float ml = sqrtf((m.x - v.x) * (m.x - v.x) + (m.y - v.y) * (m.y - v.y));
        if (ml <= limit * r) return in_triangle(p, v, a, m) || in_triangle(p, v, m, b);
    }
    return in_triangle(p, v, a, b);
}
__device__ __forceinline__ bool square_cap_hit(float2 p, float2 v, float2 d, float r) {
    const float l = sqrtf(d.x * d.x + d.y * d.y);
    if (!(l > 0.0f) || !(r > 0.0f)) return false;
    const float dx = d.x / l, dy = d.y / l, qx = p.x - v.x, qy = p.y - v.y;
    const float s = qx * dx + qy * dy, u = qx * -dy + qy * dx;
    return s >= 0.0f && s <= r && fabsf(u) <= r;
}
// The join and cap regions of a PF_STYLED path at shape-space point (px, py).  Out of
// line, with the four tables it reads as arguments (a scene reference would make the
// callers copy the whole scene to local memory).
static __device__ __forceinline__ bool join_cap_hit_v(const int4* p_info, const float* p_miter, const float4* seg_p,
                                                   const float4* seg_r, int path, float px, float py) {
    const int4 pi = __ldg(&p_info[2 * path]);
    const int pflags = __ldg(&p_info[2 * path + 1].w);
    const bool closed = pflags & PF_CLOSED;
    const int join = (pflags >> PF_JOIN_SHIFT) & 3, cap = (pflags >> PF_CAP_SHIFT) & 3;
    const float limit = __ldg(&p_miter[path]);
    const float reach = (join == JOIN_MITER ? limit : 1.0f) * 1.001f;  // join regions lie within reach * r of v
    const float2 p = make_float2(px, py);
    const int off = pi.x, n = pi.y;
    for (int k = 0; k < n; ++k) {
        const float4 a = __ldg(&seg_p[2 * (off + k)]), b = __ldg(&seg_p[2 * (off + k) + 1]);
        const float2 v = make_float2(a.x, a.y);
        const float r = __ldg(&seg_r[off + k]).x;
        if (k > 0 || closed) {
            if (join == JOIN_ROUND) continue;
            const float dx = p.x - v.x, dy = p.y - v.y;
            if (dx * dx + dy * dy > (reach * r) * (reach * r)) continue;
            const int kin = k > 0 ? k - 1 : n - 1;
            const float4 ia = __ldg(&seg_p[2 * (off + kin)]), ib = __ldg(&seg_p[2 * (off + kin) + 1]);
            if (join_hit(p, v, seg_dir1(ia, ib), seg_dir0(a, b), r, join, limit)) return true;
        } else if (cap == CAP_SQUARE) {
            const float2 d = seg_dir0(a, b);
            if (square_cap_hit(p, v, make_float2(-d.x, -d.y), r)) return true;
        }
    }
    if (!closed && cap == CAP_SQUARE && n > 0) {
        const float4 a = __ldg(&seg_p[2 * (off + n - 1)]), b = __ldg(&seg_p[2 * (off + n - 1) + 1]);
        if (square_cap_hit(p, make_float2(b.z, b.w), seg_dir1(a, b), __ldg(&seg_r[off + n - 1]).w)) return true;
    }
    return false;
}

__device__ __forceinline__ bool join_cap_hit(const DevScene& S, int path, float2 p) {
    return join_cap_hit_v(S.p_info, S.p_miter, S.seg_p, S.seg_r, path, p.x, p.y);
}
// Forward-mode derivatives of a join / cap site's polygon with respect to its vertex
// v, the control points that set the adjacent tangents (qa before, qb after the
// vertex) and the radius: 7 partials (v.x, v.y, qa.x, qa.y, qb.x, qb.y, r).  Used by the
// edge term's join / cap velocities and the prefiltered styled-stroke coverage.
struct Dl {
    float v;
    float d[7];
};
__device__ __forceinline__ Dl dl_const(float v) {
    Dl r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < 7; ++k) r.d[k] = 0.0f;
    return r;
}
__device__ __forceinline__ Dl dl_var(float v, int k) {
    Dl r = dl_const(v);
    r.d[k] = 1.0f;
    return r;
}
__device__ __forceinline__ Dl operator+(const Dl& a, const Dl& b) {
    Dl r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < 7; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
__device__ __forceinline__ Dl operator-(const Dl& a, const Dl& b) {
    Dl r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < 7; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
__device__ __forceinline__ Dl operator*(const Dl& a, const Dl& b) {
    Dl r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < 7; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
__device__ __forceinline__ Dl operator/(const Dl& a, const Dl& b) {
    Dl r;
    r.v = a.v / b.v;
#pragma unroll
    for (int k = 0; k < 7; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
__device__ __forceinline__ Dl dl_sqrt(const Dl& a) {
    Dl r;
    r.v = sqrtf(a.v);
#pragma unroll
    for (int k = 0; k < 7; ++k) r.d[k] = r.v > 0.0f ? a.d[k] * (0.5f / r.v) : 0.0f;
    return r;
}
struct DV {
    Dl x, y;
};
__device__ __forceinline__ DV dv_add(const DV& a, const DV& b) { return DV{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ DV dv_sub(const DV& a, const DV& b) { return DV{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ DV dv_scale(const DV& a, const Dl& s) { return DV{a.x * s, a.y * s}; }
__device__ __forceinline__ DV dv_unit(const DV& a) {
    const Dl l = dl_sqrt(a.x * a.x + a.y * a.y);
    return DV{a.x / l, a.y / l};
}
// Slot of the control point that seg_dir0 / seg_dir1 take (the vertex is slot 0 / 3).
__device__ __forceinline__ int seg_dir0_slot(float4 a, float4 b) {
    if (!(a.z - a.x == 0.0f && a.w - a.y == 0.0f)) return 1;
    return !(b.x - a.x == 0.0f && b.y - a.y == 0.0f) ? 2 : 3;
}
__device__ __forceinline__ int seg_dir1_slot(float4 a, float4 b) {
    if (!(b.z - b.x == 0.0f && b.w - b.y == 0.0f)) return 2;
    return !(b.z - a.z == 0.0f && b.w - a.w == 0.0f) ? 1 : 0;
}
__device__ __forceinline__ float2 seg_slot(float4 a, float4 b, int j) {
    return j == 0 ? make_float2(a.x, a.y) : j == 1 ? make_float2(a.z, a.w) : j == 2 ? make_float2(b.x, b.y)
                                                                                 : make_float2(b.z, b.w);
}
// Path point of slot j of a segment (lines and quadratics repeat their last point).
__device__ __forceinline__ int seg_slot_point(int4 meta, int j, bool closed, int pc) {
    const int idx = meta.z + (j < meta.x + 1 ? j : meta.x + 1);
    return closed ? idx % pc : idx;
}

// Nearest-segment searches keep a segment only when its distance is strictly below
// the best so far; a cubic whose lower bound exceeds that by the culling margin
// cannot be kept, so its exact solve is skipped (same argument as above).
__device__ __forceinline__ bool cubic_cannot_beat(const SegGeom& s, float2 p, bool approx, float best) {
    if (s.kind != 2 || approx || !(best < INFINITY)) return false;
    return cubic_dist_lower(p.x, p.y, s.q[0], s.q[1], s.q[2], s.q[3], s.q[4], s.q[5], s.q[6], s.q[7]) >
           best + cull_margin(s, p);
}

// ------------------------------------------------------------------ path queries
// Preorder walks with skip links move strictly forward: a descent goes to node + 1 and
// a node's skip link is node + its subtree's size (the only producer of these tables is
// the host builder, BvhBuilder in prepare.cpp; the device re-preparation in refit.cu
// rewrites bounds and leaf order, never the links), so a walk ends after at most the
// tree's node count.  The loop carries no guard: a bounds-free compare-and-select on
// every link cost the forward 10 % and the boundary evaluation 12 % on the mixed scene.
// Walks the path's BVH (preorder with skip links).  Node tests are exactly the
// crate's: ray test for winding (winding.rs:117-126), containment for strokes.
__device__ __forceinline__ int winding_path(const DevScene& S, int path, float2 p) {
    int4 pi = __ldg(&S.p_info[2 * path]);
    int n = pi.z, end = pi.z + pi.w;
    int w = 0;
    while (n < end) {
        float4 b = __ldg(&S.pn_bounds[n]);
        int4 m = __ldg(&S.pn_meta[n]);
        if (p.y < b.y || p.y > b.w || p.x > b.z) {
            n = m.x;
            continue;
        }
        if (m.z > 0) {
            for (int k = m.y; k < m.y + m.z; ++k) {
                SegGeom sg;
                load_seg(S, __ldg(&S.pl_segs[k]), sg);
                if (!ray_misses_segment(sg, p)) w += winding_segment(sg, p);
            }
            n = m.x;
        } else {
            n = n + 1;
        }
    }
    return w;
}
// Brute-force winding over the path's segments (winding.rs:52-70).
__device__ __forceinline__ int winding_path_list(const DevScene& S, int path, float2 p) {
    int4 pi = __ldg(&S.p_info[2 * path]);
    int w = 0;
    for (int k = 0; k < pi.y; ++k) {
        SegGeom sg;
        load_seg(S, pi.x + k, sg);
        if (!ray_misses_segment(sg, p)) w += winding_segment(sg, p);
    }
    return w;
}
__device__ __forceinline__ bool within_path_bvh(const DevScene& S, int path, float2 p) {  // closest.rs:20-98
    int4 pi = __ldg(&S.p_info[2 * path]);
    const int pflags = __ldg(&S.p_info[2 * path + 1].w);
    bool approx = pflags & PF_APPROX;
    int n = pi.z, end = pi.z + pi.w;
    while (n < end) {
        float4 b = __ldg(&S.pn_bounds[n]);
        int4 m = __ldg(&S.pn_meta[n]);
        if (!(p.x >= b.x && p.x <= b.z && p.y >= b.y && p.y <= b.w)) {
            n = m.x;
            continue;
        }
        if (m.z > 0) {
            for (int k = m.y; k < m.y + m.z; ++k) {
                const int sidx = __ldg(&S.pl_segs[k]);
                SegGeom sg;
                load_seg(S, sidx, sg);
                if (stroke_misses_segment(sg, p)) continue;
                if (sg.kind == 2 && !approx && stroke_far_from_cubic(sg, p)) continue;
                CPRes c = seg_closest(sg, p, approx);
                if (c.dist < seg_radius(sg, c.t) && !end_excluded(pflags, sidx - pi.x, pi.y, c.t)) return true;
            }
            n = m.x;
        } else {
            n = n + 1;
        }
    }
    return (pflags & PF_STYLED) && join_cap_hit(S, path, p);
}
__device__ __forceinline__ bool within_path_list(const DevScene& S, int path, float2 p) {  // closest.rs:228-377
    int4 pi = __ldg(&S.p_info[2 * path]);
    const int pflags = __ldg(&S.p_info[2 * path + 1].w);
    bool approx = pflags & PF_APPROX;
    for (int k = 0; k < pi.y; ++k) {
        SegGeom sg;
        load_seg(S, pi.x + k, sg);
        if (stroke_misses_segment(sg, p)) continue;
        if (sg.kind == 2 && !approx && stroke_far_from_cubic(sg, p)) continue;
        CPRes c = seg_closest(sg, p, approx);
        if (c.dist < seg_radius(sg, c.t) && !end_excluded(pflags, k, pi.y, c.t)) return true;
    }
    return (pflags & PF_STYLED) && join_cap_hit(S, path, p);
}

// ------------------------------------------------------------------ shape queries
static __device__ __noinline__ float2 closest_point_ellipse(float cx, float cy, float rx, float ry, float2 pt) {  // shape.rs:116-164
    rx = fabsf(rx);
    ry = fabsf(ry);
    const float eps = 1.0e-6f;
    if (rx < eps && ry < eps) return make_float2(cx, cy);
    if (rx < eps) return make_float2(cx, cy + clampf(pt.y - cy, -ry, ry));
    if (ry < eps) return make_float2(cx + clampf(pt.x - cx, -rx, rx), cy);
    float dx = pt.x - cx, dy = pt.y - cy;
    if (fabsf(dx) < eps && fabsf(dy) < eps) return make_float2(cx + rx, cy);
    float sx = dx < 0.0f ? -1.0f : 1.0f, sy = dy < 0.0f ? -1.0f : 1.0f;
    dx = fabsf(dx);
    dy = fabsf(dy);
    float t = dvg_atan2f(dy * rx, dx * ry);
    for (int i = 0; i < 20; ++i) {
        float s = dvg_sinf(t), c = dvg_cosf(t);
        float g = rx * dx * s - ry * dy * c + (ry * ry - rx * rx) * s * c;
        float gt = rx * dx * c + ry * dy * s + (ry * ry - rx * rx) * (c * c - s * s);
        if (fabsf(gt) < 1.0e-12f) break;
        float nx = clampf(t - g / gt, 0.0f, HALF_PI_F);
        if (fabsf(nx - t) < 1.0e-6f) {
            t = nx;
            break;
        }
        t = nx;
    }
    float s = dvg_sinf(t), c = dvg_cosf(t);
    return make_float2(cx + sx * rx * c, cy + sy * ry * s);
}
__device__ __forceinline__ float rect_signed_distance(float2 p, float4 r) {  // shape.rs:188-201
    float dx = fmaxf(fmaxf(r.x - p.x, 0.0f), p.x - r.z);
    float dy = fmaxf(fmaxf(r.y - p.y, 0.0f), p.y - r.w);
    float outside = sqrtf(dx * dx + dy * dy);
    float inside = fminf(fminf(fminf(p.x - r.x, r.z - p.x), p.y - r.y), r.w - p.y);
    return outside > 0.0f ? outside : -inside;
}
__device__ __forceinline__ float ellipse_signed_distance(float2 p, float4 prm) {  // shape.rs:204-212
    float rx = fmaxf(fabsf(fabsf(prm.z)), 1.0e-6f), ry = fmaxf(fabsf(fabsf(prm.w)), 1.0e-6f);
    float lx = p.x - prm.x, ly = p.y - prm.y;
    bool inside = (lx / rx) * (lx / rx) + (ly / ry) * (ly / ry) <= 1.0f;
    float2 c = closest_point_ellipse(prm.x, prm.y, rx, ry, p);
    float dist = len2(p.x - c.x, p.y - c.y);
    return inside ? -dist : dist;
}
// within_distance_shape (closest.rs:206-379); lp in group space.
__device__ __forceinline__ bool within_shape(const DevScene& S, int s, float2 lp, float r) {
    if (r <= 0.0f) return false;
    float2 p = shape_local_dist(S, s, lp);
    int4 si = __ldg(&S.s_info[s]);
    float4 prm = __ldg(&S.s_params[s]);
    if (si.x == K_CIRCLE) {
        float d = len2(p.x - prm.x, p.y - prm.y) - fabsf(prm.z);
        return fabsf(d) < r;
    }
    if (si.x == K_ELLIPSE) return fabsf(ellipse_signed_distance(p, prm)) < r;
    if (si.x == K_RECT) return fabsf(rect_signed_distance(p, prm)) < r;
    if (si.z < 0) return false;
    return within_path_list(S, si.z, p);
}
// winding_number_shape (winding.rs:13-48); sp in shape space.
__device__ __forceinline__ int winding_shape(const DevScene& S, int s, float2 sp, bool use_bvh) {
    int4 si = __ldg(&S.s_info[s]);
    float4 prm = __ldg(&S.s_params[s]);
    if (si.x == K_CIRCLE) {
        float r = fabsf(prm.z);
        float dx = sp.x - prm.x, dy = sp.y - prm.y;
        return (dx * dx + dy * dy) < r * r ? 1 : 0;
    }
    if (si.x == K_ELLIPSE) {
        float rx = fmaxf(fabsf(prm.z), 1.0e-6f), ry = fmaxf(fabsf(prm.w), 1.0e-6f);
        float dx = (sp.x - prm.x) / rx, dy = (sp.y - prm.y) / ry;
        return dx * dx + dy * dy < 1.0f ? 1 : 0;
    }
    if (si.x == K_RECT) return (sp.x > prm.x && sp.x < prm.z && sp.y > prm.y && sp.y < prm.w) ? 1 : 0;
    if (si.z < 0) return 0;
    int4 pi = __ldg(&S.p_info[2 * si.z]);
    if (use_bvh && pi.w > 0) return winding_path(S, si.z, sp);
    return winding_path_list(S, si.z, sp);
}
__device__ __forceinline__ bool fill_hit(int rule, int w) { return rule == 1 ? ((w < 0 ? -w : w) % 2) == 1 : w != 0; }

// ------------------------------------------------------------------ group queries (distance/api.rs)
// within_distance_bvh (api.rs:79-135) with the brute-force fallback (api.rs:15-33).
__device__ __forceinline__ bool group_within(const DevScene& S, int g, float2 lp) {
    int4 gb = __ldg(&S.g_bvh[g]);
    if (gb.y == 0) {
        for (int k = 0; k < gb.w; ++k) {
            int s = __ldg(&S.g_shape_list[gb.z + k]);
            float sw = __ldg(&S.s_stroke[s]);
            if (sw <= 0.0f) continue;
            if (within_shape(S, s, lp, sw)) return true;
        }
        return false;
    }
    int n = gb.x, end = gb.x + gb.y;
    while (n < end) {
        float4 b = __ldg(&S.gn_bounds[n]);
        int4 m = __ldg(&S.gn_meta[n]);
        if (!(lp.x >= b.x && lp.x <= b.z && lp.y >= b.y && lp.y <= b.w)) {
            n = m.x;
            continue;
        }
        if (m.z > 0) {
            for (int k = m.y; k < m.y + m.z; ++k) {
                int s = __ldg(&S.gl_shapes[k]);
                float sw = __ldg(&S.s_stroke[s]);
                if (sw <= 0.0f) continue;
                int4 si = __ldg(&S.s_info[s]);
                if (si.x == K_PATH && si.z >= 0 && __ldg(&S.p_info[2 * si.z].w) > 0) {
                    if (within_path_bvh(S, si.z, shape_local_dist(S, s, lp))) return true;
                } else if (within_shape(S, s, lp, sw)) {
                    return true;
                }
            }
            n = m.x;
        } else {
            n = n + 1;
        }
    }
    return false;
}
// is_inside_bvh (api.rs:259-309) with the brute-force fallback (api.rs:239-256).
__device__ __forceinline__ bool group_inside(const DevScene& S, int g, float2 lp, int rule) {
    int4 gb = __ldg(&S.g_bvh[g]);
    int w = 0;
    if (gb.y == 0) {
        for (int k = 0; k < gb.w; ++k) {
            int s = __ldg(&S.g_shape_list[gb.z + k]);
            w += winding_shape(S, s, shape_local_dist(S, s, lp), false);
        }
        return fill_hit(rule, w);
    }
    {
        float4 b = __ldg(&S.gn_bounds[gb.x]);
        if (!(lp.x >= b.x && lp.x <= b.z && lp.y >= b.y && lp.y <= b.w)) return false;
    }
    int n = gb.x, end = gb.x + gb.y;
    while (n < end) {
        float4 b = __ldg(&S.gn_bounds[n]);
        int4 m = __ldg(&S.gn_meta[n]);
        if (!(lp.x >= b.x && lp.x <= b.z && lp.y >= b.y && lp.y <= b.w)) {
            n = m.x;
            continue;
        }
        if (m.z > 0) {
            for (int k = m.y; k < m.y + m.z; ++k) {
                int s = __ldg(&S.gl_shapes[k]);
                w += winding_shape(S, s, shape_local_dist(S, s, lp), true);
            }
            n = m.x;
        } else {
            n = n + 1;
        }
    }
    return fill_hit(rule, w);
}

// ------------------------------------------------------------------ paints (backward/paint.rs:8-74)
__device__ __forceinline__ float4 stops_color(const DevScene& S, int so, int sc, float t) {
    if (sc <= 0) return make_float4(0, 0, 0, 0);
    if (t < __ldg(&S.stop_offsets[so])) return __ldg(&S.stop_colors[so]);
    for (int i = 0; i + 1 < sc; ++i) {
        float o0 = __ldg(&S.stop_offsets[so + i]), o1 = __ldg(&S.stop_offsets[so + i + 1]);
        if (t >= o0 && t < o1) {
            float tt = (t - o0) / (o1 - o0);
            float4 c0 = __ldg(&S.stop_colors[so + i]), c1 = __ldg(&S.stop_colors[so + i + 1]);
            return make_float4(c0.x * (1.0f - tt) + c1.x * tt, c0.y * (1.0f - tt) + c1.y * tt,
                               c0.z * (1.0f - tt) + c1.z * tt, c0.w * (1.0f - tt) + c1.w * tt);
        }
    }
    return __ldg(&S.stop_colors[so + sc - 1]);
}
__device__ __forceinline__ float paint_t(const DevScene& S, int kind, float4 pp, float2 pt) {
    if (kind == P_LINEAR) {
        float ex = pp.z - pp.x, ey = pp.w - pp.y;
        float denom = fmaxf(ex * ex + ey * ey, 1.0e-3f);
        return ((pt.x - pp.x) * ex + (pt.y - pp.y) * ey) / denom;
    }
    float nx = (pt.x - pp.x) / pp.z, ny = (pt.y - pp.y) / pp.w;
    return len2(nx, ny);
}
__device__ __forceinline__ float4 paint_color(const DevScene& S, int p, float2 pt) {
    int4 pi = __ldg(&S.paint_info[p]);
    float4 pp = __ldg(&S.paint_params[p]);
    if (pi.x == P_SOLID) return pp;
    if (pi.x == P_LINEAR || pi.x == P_RADIAL) return stops_color(S, pi.y, pi.z, paint_t(S, pi.x, pp, pt));
    return make_float4(0, 0, 0, 0);
}

// ------------------------------------------------------------------ filters (backward/filters.rs:159-239)
__device__ __forceinline__ float filter_weight(int ft, float radius, float dx, float dy) {
    if (radius <= 0.0f) return 1.0f;
    if (fabsf(dx) > radius || fabsf(dy) > radius) return 0.0f;
    if (ft == F_BOX) return 1.0f / ((2.0f * radius) * (2.0f * radius));
    if (ft == F_TENT) {
        float fx = radius - fabsf(dx), fy = radius - fabsf(dy);
        float norm = 1.0f / (radius * radius);
        return fx * fy * norm * norm;
    }
    if (ft == F_PARABOLIC) {
        float rx = 1.0f - (dx / radius) * (dx / radius), ry = 1.0f - (dy / radius) * (dy / radius);
        return (4.0f / 3.0f) * rx * (4.0f / 3.0f) * ry;
    }
    if (ft == F_HANN) {
        float ndx = (dx / (2.0f * radius)) + 0.5f, ndy = (dy / (2.0f * radius)) + 0.5f;
        float fx = 0.5f * (1.0f - dvg_cosf(2.0f * PI_F * ndx)), fy = 0.5f * (1.0f - dvg_cosf(2.0f * PI_F * ndy));
        return fx * fy * (1.0f / (radius * radius));
    }
    if (ft == F_GAUSSIAN) {  // this library's Gaussian (sigma = radius/2, square support)
        float r2 = radius * radius;
        float q = dx * dx + dy * dy;
        return (2.0f / (PI_F * r2)) * dvg_expf(-2.0f * q / r2);
    }
    return 1.0f;
}
__device__ __forceinline__ float d_filter_weight(int ft, float radius, float dx, float dy, float d_return) {
    if (ft == F_BOX) {
        float denom = 2.0f * radius;
        return denom != 0.0f ? d_return * (-2.0f) * denom / ((denom * denom) * denom) : 0.0f;
    }
    if (ft == F_TENT) {
        float fx = radius - fabsf(dx), fy = radius - fabsf(dy);
        float norm = 1.0f / (radius * radius);
        float d_fx = d_return * fy * norm, d_fy = d_return * fx * norm, d_norm = d_return * fx * fy;
        float r2 = radius * radius;
        return radius != 0.0f ? d_fx + d_fy + (-4.0f) * d_norm / ((r2 * r2) * radius) : 0.0f;
    }
    if (ft == F_PARABOLIC) {
        float r3 = radius * radius * radius;
        return r3 != 0.0f ? -(2.0f * dx * dx + 2.0f * dy * dy) / r3 : 0.0f;
    }
    if (ft == F_HANN) {
        float ndx = (dx / (2.0f * radius)) + 0.5f, ndy = (dy / (2.0f * radius)) + 0.5f;
        float fx = 0.5f * (1.0f - dvg_cosf(2.0f * PI_F * ndx)), fy = 0.5f * (1.0f - dvg_cosf(2.0f * PI_F * ndy));
        float norm = 1.0f / (radius * radius);
        float d_fx = d_return * fy * norm, d_fy = d_return * fx * norm, d_norm = d_return * fx * fy;
        float d_ndx = d_fx * 0.5f * dvg_sinf(2.0f * PI_F * ndx) * (2.0f * PI_F);
        float d_ndy = d_fy * 0.5f * dvg_sinf(2.0f * PI_F * ndy) * (2.0f * PI_F);
        float tr = 2.0f * radius;
        return d_ndx * (-2.0f * dx / (tr * tr)) + d_ndy * (-2.0f * dy / (tr * tr)) +
               (-2.0f) * d_norm / ((radius * radius) * radius);
    }
    if (ft == F_GAUSSIAN) {
        float r2 = radius * radius;
        float q = dx * dx + dy * dy;
        float w = (2.0f / (PI_F * r2)) * dvg_expf(-2.0f * q / r2);
        return radius != 0.0f ? d_return * w * (4.0f * q / (r2 * radius) - 2.0f / radius) : 0.0f;
    }
    return 0.0f;
}

// ------------------------------------------------------------------ random numbers
// PCG32 exactly as src/renderer/rng.rs:16-43 (native 64-bit arithmetic).
struct Pcg32 {
    uint64_t state, inc;
    __device__ Pcg32(uint64_t idx, uint64_t seed) {
        state = 0;
        inc = ((idx + 1) << 1) | 1;
        next();
        state += 0x853c49e6748fea9bULL + seed;
        next();
    }
    __device__ __forceinline__ uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + (inc | 1);
        uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return __funnelshift_r(xs, xs, rot);
    }
    __device__ __forceinline__ float next_f32() {
        uint32_t u = next();
        return __uint_as_float((u >> 9) | 0x3f800000u) - 1.0f;
    }
};
// Philox4x32-10 (Salmon et al., SC'11); counter (idx_lo, idx_hi, 0, 0), key (seed, 0).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
__device__ __forceinline__ float unit_from_u32(uint32_t u) { return (float)(u >> 9) * (1.0f / 8388608.0f); }

// Sample position (src/backward/render.rs:95-111; idx = ((y*W+x)*sy_n+sy)*sx_n+sx).
__device__ __forceinline__ float2 sample_pos(int x, int y, int sx, int sy, int sxn, int syn, int W, uint32_t seed,
                                             bool jitter) {
    float rx = 0.5f, ry = 0.5f;
    if (jitter) {
        uint64_t idx = (((uint64_t)y * W + x) * syn + sy) * sxn + sx;
        Pcg32 rng(idx, (uint64_t)seed);
        rx = rng.next_f32();
        ry = rng.next_f32();
    }
    return make_float2((float)x + ((float)sx + rx) / (float)sxn, (float)y + ((float)sy + ry) / (float)syn);
}

__device__ __forceinline__ float4 background_premul(const DevScene& S, int pixel) {  // background.rs:7-26
    if (S.bg_image) {
        const float* b = S.bg_image + 4 * (size_t)pixel;
        return make_float4(b[0] * b[3], b[1] * b[3], b[2] * b[3], b[3]);
    }
    return make_float4(S.bg[0] * S.bg[3], S.bg[1] * S.bg[3], S.bg[2] * S.bg[3], S.bg[3]);
}

// Tile lookup for an arbitrary canvas point (edge tiles extend to infinity in binning).
__device__ __forceinline__ int tile_of(const DevScene& S, float2 p) {
    int tx = f2i(floorf(p.x / (float)TILE)), ty = f2i(floorf(p.y / (float)TILE));
    tx = tx < 0 ? 0 : (tx >= S.tiles_x ? S.tiles_x - 1 : tx);
    ty = ty < 0 ? 0 : (ty >= S.tiles_y ? S.tiles_y - 1 : ty);
    return ty * S.tiles_x + tx;
}

// Premultiplied over (src/backward/sampling.rs:153-154 / forward.rs:370-377).
__device__ __forceinline__ void over(float4& acc, float4 c) {
    float a = c.w, inv = 1.0f - a;
    acc.x = acc.x * inv + c.x * a;
    acc.y = acc.y * inv + c.y * a;
    acc.z = acc.z * inv + c.z * a;
    acc.w = acc.w * inv + a;
}

// ------------------------------------------------------------------ gradients
struct GradPtrs {
    float* d_shape_params;
    float* d_shape_transform;
    float* d_shape_stroke_width;
    float* d_points;
    float* d_thickness;
    float* d_group_transform;
    float* d_paint_params;
    float* d_stop_offsets;
    float* d_stop_colors;
    float* d_filter_radius;
    float* d_background;
    float* d_background_image;
    float* d_translation;
};

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ void add_if(float* p, float v) {
    if (v != 0.0f) atomicAdd(p, v);
}

// d_sample_paint for gradient paints (backward/paint.rs:91-277), split in the terms one
// sample adds and where they go.  stop: the stop whose colour takes c0 (an interval
// [o_stop, o_stop+1) also gives c1 to stop + 1, the two stop-offset terms when the
// interval has a width, and the paint-parameter terms); -1: nothing to add.
struct PaintGradTerms {
    int stop;
    bool interval, has_off;
    float4 c0, c1;
    float off0, off1;
    float4 pp;
};
static __device__ __forceinline__ PaintGradTerms gradient_paint_terms(const DevScene& S, int p, float2 pt, float4 dc,
                                                                     float2* dtr) {
    PaintGradTerms r;
    r.stop = -1;
    r.interval = r.has_off = false;
    r.c0 = r.c1 = r.pp = make_float4(0, 0, 0, 0);
    r.off0 = r.off1 = 0.0f;
    int4 pi = __ldg(&S.paint_info[p]);
    float4 pp = __ldg(&S.paint_params[p]);
    int so = pi.y, sc = pi.z;
    if (sc <= 0) return r;
    float t, denom = 0.0f, offx = 0.0f, offy = 0.0f, nx = 0.0f, ny = 0.0f;
    if (pi.x == P_LINEAR) {
        float ex = pp.z - pp.x, ey = pp.w - pp.y;
        denom = fmaxf(ex * ex + ey * ey, 1.0e-3f);
        t = ((pt.x - pp.x) * ex + (pt.y - pp.y) * ey) / denom;
    } else {
        offx = pt.x - pp.x;
        offy = pt.y - pp.y;
        nx = offx / pp.z;
        ny = offy / pp.w;
        t = len2(nx, ny);
    }
    if (t < __ldg(&S.stop_offsets[so])) {
        r.stop = so;
        r.c0 = dc;
        return r;
    }
    for (int i = 0; i + 1 < sc; ++i) {
        float o0 = __ldg(&S.stop_offsets[so + i]), o1 = __ldg(&S.stop_offsets[so + i + 1]);
        if (t >= o0 && t < o1) {
            float tt = (t - o0) / (o1 - o0);
            float4 c0 = __ldg(&S.stop_colors[so + i]), c1 = __ldg(&S.stop_colors[so + i + 1]);
            r.stop = so + i;
            r.interval = true;
            r.c0 = make_float4(dc.x * (1.0f - tt), dc.y * (1.0f - tt), dc.z * (1.0f - tt), dc.w * (1.0f - tt));
            r.c1 = make_float4(dc.x * tt, dc.y * tt, dc.z * tt, dc.w * tt);
            float d_tt = dc.x * (c1.x - c0.x) + dc.y * (c1.y - c0.y) + dc.z * (c1.z - c0.z) + dc.w * (c1.w - c0.w);
            float dof = o1 - o0;
            if (fabsf(dof) > 0.0f) {
                r.has_off = true;
                r.off0 = d_tt * (tt - 1.0f) / dof;
                r.off1 = -d_tt * tt / dof;
            }
            float d_t = d_tt / dof;
            if (pi.x == P_LINEAR) {
                float bx = d_t * (-(pt.x - pp.x) - (pp.z - pp.x)) / denom;
                float by = d_t * (-(pt.y - pp.y) - (pp.w - pp.y)) / denom;
                float ex = d_t * (pt.x - pp.x) / denom;
                float ey = d_t * (pt.y - pp.y) / denom;
                float d_l = -d_t * t / denom;
                float lx = pp.z - pp.x, ly = pp.w - pp.y;
                if (lx * lx + ly * ly > 1.0e-3f) {
                    float ax = pp.x - pp.z, ay = pp.y - pp.w;
                    r.pp = make_float4(bx + 2.0f * d_l * ax, by + 2.0f * d_l * ay, ex + 2.0f * d_l * lx,
                                       ey + 2.0f * d_l * ly);
                } else {
                    r.pp = make_float4(bx, by, ex, ey);
                }
                dtr->x += bx + ex;
                dtr->y += by + ey;
            } else {
                // d_length(normalized, d_t) (backward/math.rs:33-41)
                float l = sqrtf(nx * nx + ny * ny);
                float dnx = 0.0f, dny = 0.0f;
                if (l != 0.0f) {
                    float dls = 0.5f * d_t / l;
                    dnx = nx * (2.0f * dls);
                    dny = ny * (2.0f * dls);
                }
                float dox = dnx / pp.z, doy = dny / pp.w;
                float drx = -dnx * offx / (pp.z * pp.z), dry = -dny * offy / (pp.w * pp.w);
                r.pp = make_float4(-dox, -doy, drx, dry);
                dtr->x += -dox;
                dtr->y += -doy;
            }
            return r;
        }
    }
    r.stop = so + sc - 1;
    r.c0 = dc;
    return r;
}
static __device__ __forceinline__ void add4_if(float* d, float4 v) {
    add_if(d + 0, v.x);
    add_if(d + 1, v.y);
    add_if(d + 2, v.z);
    add_if(d + 3, v.w);
}
static __device__ __forceinline__ void add_paint_terms(const GradPtrs& G, int p, const PaintGradTerms& r) {
    if (r.stop < 0) return;
    float* a0 = G.d_stop_colors + 4 * r.stop;
    add4_if(a0, r.c0);
    if (!r.interval) return;
    add4_if(a0 + 4, r.c1);
    if (r.has_off) {
        add_if(G.d_stop_offsets + r.stop, r.off0);
        add_if(G.d_stop_offsets + r.stop + 1, r.off1);
    }
    add4_if(G.d_paint_params + 4 * p, r.pp);
}
__device__ __forceinline__ float4 warp_sum4(float4 v) {
    return make_float4(warp_sum(v.x), warp_sum(v.y), warp_sum(v.z), warp_sum(v.w));
}
// d_sample_paint of a gradient paint for a whole warp whose lanes share paint p (all
// 32 lanes call it; `has`: this lane has a contribution).  When every contributing lane adds to the same stop
// (or stop interval) the terms are summed over the warp and one lane adds them: 1
// atomic per term instead of one per lane, all of them on one cache line.  The same
// terms, summed in another order.
static __device__ void d_gradient_paint_warp(const DevScene& S, const GradPtrs& G, int p, float2 pt, float4 dc,
                                             bool has, float2* dtr) {
    PaintGradTerms r;
    r.stop = -1;
    if (has) r = gradient_paint_terms(S, p, pt, dc, dtr);
    const int key = r.stop < 0 ? -1 : 2 * r.stop + (r.interval ? 1 : 0);
    const int kmax = __reduce_max_sync(0xffffffffu, key);
    const int kmin = __reduce_min_sync(0xffffffffu, key < 0 ? 0x7fffffff : key);
    if (kmax < 0) return;
    if (kmin != kmax) {  // lanes in different stop intervals
        add_paint_terms(G, p, r);
        return;
    }
    if (r.stop < 0) {
        r.c0 = r.c1 = r.pp = make_float4(0, 0, 0, 0);
        r.off0 = r.off1 = 0.0f;
    }
    const bool interval = (kmax & 1) != 0;
    const float4 c0 = warp_sum4(r.c0);
    float4 c1 = make_float4(0, 0, 0, 0), pp4 = make_float4(0, 0, 0, 0);
    float o0 = 0.0f, o1 = 0.0f;
    if (interval) {
        c1 = warp_sum4(r.c1);
        pp4 = warp_sum4(r.pp);
        o0 = warp_sum(r.off0);
        o1 = warp_sum(r.off1);
    }
    if ((threadIdx.x & 31) != 0) return;
    const int stop = kmax >> 1;
    float* a0 = G.d_stop_colors + 4 * stop;
    add4_if(a0, c0);
    if (!interval) return;
    add4_if(a0 + 4, c1);
    add_if(G.d_stop_offsets + stop, o0);  // zero sums (an interval without width) add nothing
    add_if(G.d_stop_offsets + stop + 1, o1);
    add4_if(G.d_paint_params + 4 * p, pp4);
}

// ------------------------------------------------------------------ filtered splat / gather
// Adds the sample's premultiplied colour times the filter weight (and the weight)
// to every pixel of its (2*ri+1)^2 footprint: into the CTA's shared tile+halo
// accumulator when it fits, else straight to global memory.
__device__ __forceinline__ void splat_sample(const DevScene& S, int x, int y, int tx, int ty, int ri, int HW,
                                             bool use_sm, float2 pt, float4 acc, float* sm, float* accum,
                                             float* wsum) {
    for (int dy = -ri; dy <= ri; ++dy)
        for (int dx = -ri; dx <= ri; ++dx) {
            int xx = x + dx, yy = y + dy;
            if (xx < 0 || yy < 0 || xx >= S.width || yy >= S.height) continue;
            float w = filter_weight(S.filter_type, S.filter_radius, (float)xx + 0.5f - pt.x, (float)yy + 0.5f - pt.y);
            if (!(w > 0.0f)) continue;
            if (use_sm) {
                int li = (yy - (ty * TILE - ri)) * HW + (xx - (tx * TILE - ri));
                float* c = sm + 5 * li;
                atomicAdd(c + 0, acc.x * w);
                atomicAdd(c + 1, acc.y * w);
                atomicAdd(c + 2, acc.z * w);
                atomicAdd(c + 3, acc.w * w);
                atomicAdd(c + 4, w);
            } else {
                size_t p = (size_t)yy * S.width + xx;
                atomicAdd(accum + 4 * p + 0, acc.x * w);
                atomicAdd(accum + 4 * p + 1, acc.y * w);
                atomicAdd(accum + 4 * p + 2, acc.z * w);
                atomicAdd(accum + 4 * p + 3, acc.w * w);
                atomicAdd(wsum + p, w);
            }
        }
}
// Flushes the CTA's tile+halo accumulator to global memory (one atomic per value).
__device__ __forceinline__ void flush_splat(const DevScene& S, int tx, int ty, int ri, int HW, const float* sm,
                                            float* accum, float* wsum) {
    for (int i = threadIdx.x; i < HW * HW; i += blockDim.x) {
        const float* c = sm + 5 * i;
        if (c[4] == 0.0f) continue;
        int xx = tx * TILE - ri + i % HW, yy = ty * TILE - ri + i / HW;
        if (xx < 0 || yy < 0 || xx >= S.width || yy >= S.height) continue;
        size_t p = (size_t)yy * S.width + xx;
        atomicAdd(accum + 4 * p + 0, c[0]);
        atomicAdd(accum + 4 * p + 1, c[1]);
        atomicAdd(accum + 4 * p + 2, c[2]);
        atomicAdd(accum + 4 * p + 3, c[3]);
        atomicAdd(wsum + p, c[4]);
    }
}
// gather_d_color (src/backward/filters.rs:70-103)
__device__ __forceinline__ float4 gather_d_color(const DevScene& S, const float* d_render, const float* wsum,
                                                 float2 ps) {
    float4 out = make_float4(0, 0, 0, 0);
    const int px = f2i(floorf(ps.x)), py = f2i(floorf(ps.y)), ri = S.filter_ri;
    for (int dy = -ri; dy <= ri; ++dy)
        for (int dx = -ri; dx <= ri; ++dx) {
            int xx = px + dx, yy = py + dy;
            if (xx < 0 || yy < 0 || xx >= S.width || yy >= S.height) continue;
            float w = filter_weight(S.filter_type, S.filter_radius, (float)xx + 0.5f - ps.x, (float)yy + 0.5f - ps.y);
            size_t q = (size_t)yy * S.width + xx;
            float ws = wsum[q];
            if (ws > 0.0f) {
                float4 d = reinterpret_cast<const float4*>(d_render)[q];
                float k = w / ws;
                out.x += k * d.x;
                out.y += k * d.y;
                out.z += k * d.z;
                out.w += k * d.w;
            }
        }
    return out;
}
// accumulate_filter_gradient (src/backward/filters.rs:106-156) for one sample; returns d radius.
__device__ __forceinline__ float filter_radius_adjoint(const DevScene& S, const float* d_render, const float* wsum,
                                                       float2 ps, float4 color) {
    float dradius = 0.0f;
    const int px = f2i(floorf(ps.x)), py = f2i(floorf(ps.y)), ri = S.filter_ri;
    for (int dy = -ri; dy <= ri; ++dy)
        for (int dx = -ri; dx <= ri; ++dx) {
            int xx = px + dx, yy = py + dy;
            if (xx < 0 || yy < 0 || xx >= S.width || yy >= S.height) continue;
            size_t q = (size_t)yy * S.width + xx;
            float ws = wsum[q];
            if (ws <= 0.0f) continue;
            float fxc = (float)xx + 0.5f - ps.x, fyc = (float)yy + 0.5f - ps.y;
            float w = filter_weight(S.filter_type, S.filter_radius, fxc, fyc);
            if (w <= 0.0f) continue;
            float4 d = reinterpret_cast<const float4*>(d_render)[q];
            float dt = d.x * color.x + d.y * color.y + d.z * color.z + d.w * color.w;
            float denom = ws * ws;
            float dw = denom > 0.0f ? (dt * ws - w * dt * (ws - w)) / denom : 0.0f;
            if (dw != 0.0f) dradius += d_filter_weight(S.filter_type, S.filter_radius, fxc, fyc, dw);
        }
    return dradius;
}

}  // namespace dvgb
