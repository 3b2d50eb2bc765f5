// oracle.cpp — CPU oracle (test infrastructure only; see oracle.h).
//
// Restates the diffvg-rs crate's CPU arithmetic function by function.  Each
// function names the crate file:line it follows.  Arithmetic is f32 where the
// crate uses f32 and f64 where the crate casts to f64; the file is compiled
// with -ffp-contract=off so no multiply-add is fused (Rust never fuses).
// Where the crate has no CPU code (the forward image), the GPU pipeline
// semantics of src/gpu/kernels/forward.rs are followed (see oracle_render).
//
// Parity: pinned by the crate's known-answer tests (tests/test_oracle_kat.py
// restates src/distance/tests.rs and src/geometry.rs:509-519); render and
// gradients are "parity unpinned" (no crate tests, crate not buildable here).

#include "oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace orc {

// Work accounting for the compute roofline (built only into oracle/_build/liboracle_ops.so,
// -DORACLE_COUNT_OPS; a no-op in the oracle proper).  OPS(n) adds the floating-point
// operations of the straight-line block it follows: one per f32 or f64 add, subtract,
// multiply, divide and square root, one per libm call (acos, cos, pow, sin, atan2);
// negation, comparisons, abs, min / max and conversions count zero.
#ifdef ORACLE_COUNT_OPS
static thread_local uint64_t g_ops = 0;
#define OPS(n) (g_ops += (uint64_t)(n))
#else
#define OPS(n) ((void)0)
#endif

static const float PI_F = 3.14159265358979323846f;       // core::f32::consts::PI
static const float FRAC_PI_2_F = 1.57079632679489661923f;  // core::f32::consts::FRAC_PI_2
static const float INF_F = std::numeric_limits<float>::infinity();

// ---------------------------------------------------------------- math (src/math.rs)
struct V2 {
    float x, y;
};
static inline V2 mk(float x, float y) { return V2{x, y}; }
static inline V2 operator+(V2 a, V2 b) { return V2{a.x + b.x, a.y + b.y}; }
static inline V2 operator-(V2 a, V2 b) { return V2{a.x - b.x, a.y - b.y}; }
static inline V2 operator*(V2 a, float s) { return V2{a.x * s, a.y * s}; }
static inline V2 operator/(V2 a, float s) { return V2{a.x / s, a.y / s}; }
static inline V2& operator+=(V2& a, V2 b) {
    a.x += b.x;
    a.y += b.y;
    return a;
}
static inline V2& operator-=(V2& a, V2 b) {
    a.x -= b.x;
    a.y -= b.y;
    return a;
}
static inline bool operator==(V2 a, V2 b) { return a.x == b.x && a.y == b.y; }
static inline float dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }        // math.rs:24-26
static inline float cross(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }      // math.rs:29-31
static inline float length_sq(V2 a) { return dot(a, a); }                    // math.rs:39-41
static inline float length(V2 a) { return std::sqrt(length_sq(a)); }        // math.rs:34-36
static inline V2 vmin(V2 a, V2 b) { return V2{std::fmin(a.x, b.x), std::fmin(a.y, b.y)}; }
static inline V2 vmax(V2 a, V2 b) { return V2{std::fmax(a.x, b.x), std::fmax(a.y, b.y)}; }
static inline V2 lerp(V2 a, V2 b, float t) {  // math.rs:54-56
    return V2{a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t};
}
// Rust f32::clamp (panics on min>max, keeps NaN).
static inline float clampf(float v, float lo, float hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}
static inline double clampd(double v, double lo, double hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}
// Rust `f as i32`: saturating, NaN -> 0.
static inline int32_t to_i32(float f) {
    if (std::isnan(f)) return 0;
    if (f >= 2147483647.0f) return INT32_MAX;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (int32_t)f;
}

struct V4 {
    float x, y, z, w;
};
static inline float dot4(V4 a, V4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

struct M3 {
    float m[3][3];
};
static inline M3 identity3() {
    M3 r;
    std::memset(&r, 0, sizeof(r));
    r.m[0][0] = r.m[1][1] = r.m[2][2] = 1.0f;
    return r;
}
static inline M3 zero3() {
    M3 r;
    std::memset(&r, 0, sizeof(r));
    return r;
}
static inline M3 mul3(const M3& a, const M3& b) {  // math.rs:185-195
    M3 o;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            o.m[r][c] = a.m[r][0] * b.m[0][c] + a.m[r][1] * b.m[1][c] + a.m[r][2] * b.m[2][c];
    return o;
}
static inline V2 xform_pt(const M3& t, V2 v) {  // math.rs:198-202
    float x = t.m[0][0] * v.x + t.m[0][1] * v.y + t.m[0][2];
    float y = t.m[1][0] * v.x + t.m[1][1] * v.y + t.m[1][2];
    return V2{x, y};
}
static const float M3_EPS = 1.0e-6f;  // math.rs:6
static inline bool is_identity(const M3& t) {  // math.rs:212-222
    return std::fabs(t.m[0][0] - 1.0f) < M3_EPS && std::fabs(t.m[0][1]) < M3_EPS &&
           std::fabs(t.m[0][2]) < M3_EPS && std::fabs(t.m[1][0]) < M3_EPS &&
           std::fabs(t.m[1][1] - 1.0f) < M3_EPS && std::fabs(t.m[1][2]) < M3_EPS &&
           std::fabs(t.m[2][0]) < M3_EPS && std::fabs(t.m[2][1]) < M3_EPS &&
           std::fabs(t.m[2][2] - 1.0f) < M3_EPS;
}
static inline float max_scale(const M3& t) {  // math.rs:250-266
    float sx = std::sqrt(t.m[0][0] * t.m[0][0] + t.m[1][0] * t.m[1][0]);
    float sy = std::sqrt(t.m[0][1] * t.m[0][1] + t.m[1][1] * t.m[1][1]);
    return std::fmax(sx, sy);
}
static inline bool inverse3(const M3& t, M3* out) {  // math.rs:269-290
    float a = t.m[0][0], b = t.m[0][1], c = t.m[1][0], d = t.m[1][1];
    float tx = t.m[0][2], ty = t.m[1][2];
    float det = a * d - b * c;
    if (std::fabs(det) < M3_EPS) return false;
    float inv_det = 1.0f / det;
    float m00 = d * inv_det, m01 = -b * inv_det, m10 = -c * inv_det, m11 = a * inv_det;
    float m02 = -(m00 * tx + m01 * ty);
    float m12 = -(m10 * tx + m11 * ty);
    M3 r;
    r.m[0][0] = m00; r.m[0][1] = m01; r.m[0][2] = m02;
    r.m[1][0] = m10; r.m[1][1] = m11; r.m[1][2] = m12;
    r.m[2][0] = 0.0f; r.m[2][1] = 0.0f; r.m[2][2] = 1.0f;
    *out = r;
    return true;
}
// distance/utils.rs:7-16 (identity shortcut; singular -> unchanged point)
static inline V2 xform_inv_dist(const M3& t, V2 pt) {
    if (is_identity(t)) return pt;
    M3 inv;
    if (inverse3(t, &inv)) return xform_pt(inv, pt);
    return pt;
}
// backward/math.rs:131-135 (no identity shortcut; singular -> identity)
static inline V2 xform_inv_bwd(const M3& t, V2 pt) {
    M3 inv;
    if (!inverse3(t, &inv)) inv = identity3();
    return xform_pt(inv, pt);
}

// ---------------------------------------------------------------- scene model (src/scene.rs)
struct Color {
    float r, g, b, a;
};
struct Stop {
    float offset;
    Color color;
};
struct Paint {
    uint32_t kind;  // DVG_PAINT_*
    float p[4];
    std::vector<Stop> stops;
};
struct PathG {  // geometry.rs:78-89
    std::vector<uint8_t> ncp;
    std::vector<V2> pts;
    bool has_thick = false;
    std::vector<float> thick;
    bool closed = false;
    bool approx = false;
    uint32_t point_base = 0;  // offset of pts[0] in the flat description
};
struct Shape {  // scene.rs:184-197
    uint32_t kind;
    float prm[4];
    PathG path;
    M3 transform;
    float stroke_width;
    uint32_t join;
    float miter;
    uint32_t cap = DVG_CAP_ROUND;
};
struct Group {  // scene.rs:215-230
    std::vector<size_t> shape_ids;
    int fill = -1, stroke = -1;  // paint indices
    uint32_t fill_rule = 0;
    M3 s2c, c2s;
};
struct Scene {  // scene.rs:261-276
    uint32_t w = 0, h = 0;
    std::vector<Shape> shapes;
    std::vector<Group> groups;
    std::vector<Paint> paints;
    std::vector<uint32_t> paint_stop_base;
    Color bg{0, 0, 0, 0};
    bool has_bg_img = false;
    std::vector<float> bg_img;
    uint32_t filter_type = 0;
    float filter_radius = 0.5f;
};

static M3 load_m3(const float* p) {
    M3 r;
    for (int i = 0; i < 9; ++i) r.m[i / 3][i % 3] = p[i];
    return r;
}

static Scene decode(const dvg_scene_desc* d) {
    Scene s;
    s.w = d->width;
    s.h = d->height;
    s.bg = Color{d->background[0], d->background[1], d->background[2], d->background[3]};
    if (d->background_image) {
        s.has_bg_img = true;
        s.bg_img.assign(d->background_image, d->background_image + (size_t)d->width * d->height * 4);
    }
    s.filter_type = d->filter_type;
    s.filter_radius = d->filter_radius;
    s.shapes.resize(d->num_shapes);
    for (uint32_t i = 0; i < d->num_shapes; ++i) {
        Shape& sh = s.shapes[i];
        sh.kind = d->shape_kind[i];
        for (int k = 0; k < 4; ++k) sh.prm[k] = d->shape_params[4 * i + k];
        sh.transform = load_m3(d->shape_transform + 9 * i);
        sh.stroke_width = d->shape_stroke_width[i];
        sh.join = d->shape_stroke_join ? d->shape_stroke_join[i] : (uint32_t)DVG_JOIN_ROUND;
        sh.miter = d->shape_miter_limit ? d->shape_miter_limit[i] : 4.0f;
        sh.cap = d->shape_stroke_cap ? d->shape_stroke_cap[i] : (uint32_t)DVG_CAP_ROUND;
        if (sh.kind == DVG_SHAPE_PATH) {
            uint32_t co = d->path_ctrl_offset[i], cc = d->path_ctrl_count[i];
            uint32_t po = d->path_point_offset[i], pc = d->path_point_count[i];
            uint32_t fl = d->path_flags[i];
            sh.path.ncp.assign(d->num_control_points + co, d->num_control_points + co + cc);
            sh.path.pts.resize(pc);
            for (uint32_t k = 0; k < pc; ++k)
                sh.path.pts[k] = mk(d->points[2 * (po + k)], d->points[2 * (po + k) + 1]);
            sh.path.closed = (fl & DVG_PATH_CLOSED) != 0;
            sh.path.approx = (fl & DVG_PATH_DISTANCE_APPROX) != 0;
            sh.path.has_thick = (fl & DVG_PATH_HAS_THICKNESS) != 0 && d->thickness != nullptr;
            if (sh.path.has_thick) sh.path.thick.assign(d->thickness + po, d->thickness + po + pc);
            sh.path.point_base = po;
        }
    }
    s.paints.resize(d->num_paints);
    s.paint_stop_base.resize(d->num_paints);
    for (uint32_t i = 0; i < d->num_paints; ++i) {
        Paint& p = s.paints[i];
        p.kind = d->paint_kind[i];
        for (int k = 0; k < 4; ++k) p.p[k] = d->paint_params[4 * i + k];
        uint32_t so = d->paint_stop_offset ? d->paint_stop_offset[i] : 0;
        uint32_t sc = d->paint_stop_count ? d->paint_stop_count[i] : 0;
        s.paint_stop_base[i] = so;
        for (uint32_t k = 0; k < sc; ++k) {
            Stop st;
            st.offset = d->stop_offsets[so + k];
            const float* c = d->stop_colors + 4 * (so + k);
            st.color = Color{c[0], c[1], c[2], c[3]};
            p.stops.push_back(st);
        }
    }
    s.groups.resize(d->num_groups);
    for (uint32_t g = 0; g < d->num_groups; ++g) {
        Group& gr = s.groups[g];
        uint32_t so = d->group_shape_offset[g], sc = d->group_shape_count[g];
        for (uint32_t k = 0; k < sc; ++k) gr.shape_ids.push_back(d->group_shape_ids[so + k]);
        gr.fill = d->group_fill_paint[g];
        gr.stroke = d->group_stroke_paint[g];
        gr.fill_rule = d->group_fill_rule[g];
        gr.s2c = load_m3(d->group_shape_to_canvas + 9 * g);
        gr.c2s = load_m3(d->group_canvas_to_shape + 9 * g);
    }
    return s;
}

// ---------------------------------------------------------------- path helpers (src/path_utils.rs)
static bool path_point(const PathG& p, size_t index, V2* out) {  // path_utils.rs:7-16
    size_t total = p.pts.size();
    if (total == 0) return false;
    if (p.closed) {
        *out = p.pts[index % total];
        return true;
    }
    if (index >= total) return false;
    *out = p.pts[index];
    return true;
}
static bool path_point_radius(const PathG& p, size_t index, float default_radius, V2* pt,
                              float* r) {  // path_utils.rs:19-41 (thickness_scale = 1)
    if (!path_point(p, index, pt)) return false;
    size_t total = p.pts.size();
    size_t idx = p.closed ? index % total : index;
    if (p.has_thick && idx < p.thick.size())
        *r = p.thick[idx] * 1.0f;
    else
        *r = default_radius;
    return true;
}
// distance/utils.rs:24-45
static bool path_segment_points(const PathG& p, size_t point_id, uint8_t nc, V2* q, size_t* next) {
    if (!path_point(p, point_id, &q[0])) return false;
    if (!path_point(p, point_id + 1, &q[1])) return false;
    if (nc == 0) {
        q[2] = q[1];
        q[3] = q[1];
        *next = point_id + 1;
        return true;
    }
    if (nc == 1) {
        if (!path_point(p, point_id + 2, &q[2])) return false;
        q[3] = q[2];
        *next = point_id + 2;
        return true;
    }
    if (nc == 2) {
        if (!path_point(p, point_id + 2, &q[2])) return false;
        if (!path_point(p, point_id + 3, &q[3])) return false;
        *next = point_id + 3;
        return true;
    }
    return false;
}

// ---------------------------------------------------------------- polynomial roots (distance/utils.rs:48-123)
static bool solve_quadratic(double a, double b, double c, double t[2]) {
    const double eps = 1.0e-12;
    if (std::fabs(a) < eps) {
        if (std::fabs(b) < eps) return false;
        double root = -c / b;
        OPS(1);
        t[0] = root;
        t[1] = root;
        return true;
    }
    double discrim = b * b - 4.0 * a * c;
    OPS(4);
    if (discrim < 0.0) return false;
    double root = std::sqrt(discrim);
    OPS(1);
    if (std::fabs(root) < eps) {
        double r = -0.5 * b / a;
        OPS(2);
        t[0] = r;
        t[1] = r;
        return true;
    }
    double q = (b < 0.0) ? -0.5 * (b - root) : -0.5 * (b + root);
    OPS(2);
    if (std::fabs(q) < eps) {
        double inv = 0.5 / a;
        t[0] = (-b - root) * inv;
        t[1] = (-b + root) * inv;
        OPS(5);
    } else {
        t[0] = q / a;
        t[1] = c / q;
        OPS(2);
    }
    if (t[0] > t[1]) std::swap(t[0], t[1]);
    return true;
}
static double cbrt_ref(double x) {  // distance/utils.rs:115-123
    if (x > 0.0) return OPS(1), std::pow(x, 1.0 / 3.0);
    if (x < 0.0) return OPS(1), -std::pow(-x, 1.0 / 3.0);
    return 0.0;
}
static int solve_cubic(double a, double b, double c, double d, double t[3]) {
    if (std::fabs(a) < 1.0e-6) {
        double roots[2] = {0.0, 0.0};
        if (solve_quadratic(b, c, d, roots)) {
            t[0] = roots[0];
            t[1] = roots[1];
            return 2;
        }
        return 0;
    }
    b = b / a;
    c = c / a;
    d = d / a;
    double q = (b * b - 3.0 * c) / 9.0;
    double r = (2.0 * b * b * b - 9.0 * b * c + 27.0 * d) / 54.0;
    OPS(3 + 4 + 9 + 3);  // normalise, q, r, the discriminant test r*r < q*q*q
    if (r * r < q * q * q) {
        double theta = std::acos(r / std::sqrt(q * q * q));
        t[0] = -2.0 * std::sqrt(q) * std::cos(theta / 3.0) - b / 3.0;
        t[1] = -2.0 * std::sqrt(q) * std::cos((theta + 2.0 * M_PI) / 3.0) - b / 3.0;
        t[2] = -2.0 * std::sqrt(q) * std::cos((theta - 2.0 * M_PI) / 3.0) - b / 3.0;
        OPS(5 + 7 + 8 + 8);
        return 3;
    }
    double a_root = (r > 0.0) ? -cbrt_ref(r + std::sqrt(r * r - q * q * q))
                              : cbrt_ref(-r + std::sqrt(r * r - q * q * q));
    double b_root = (std::fabs(a_root) > 1.0e-6) ? (OPS(1), q / a_root) : 0.0;
    t[0] = (a_root + b_root) - b / 3.0;
    OPS(6 + 3);  // r*r - q*q*q, sqrt, +-r; (a + b) - b/3
    return 1;
}

// ---------------------------------------------------------------- curve distance (distance/curve.rs)
struct CP {  // (closest point, t, dist)
    V2 cp;
    float t;
    float dist;
};
static inline void distance_to_segment(V2 pt, V2 a, V2 b, float* dist, V2* cp, float* t) {
    V2 ab = b - a;  // curve.rs:10-21
    float denom = dot(ab, ab);
    OPS(5);
    if (denom <= 1.0e-10f) {
        *dist = length(pt - a);
        OPS(6);
        *cp = a;
        *t = 0.0f;
        return;
    }
    float tt = clampf(dot(pt - a, ab) / denom, 0.0f, 1.0f);
    V2 c = a + ab * tt;
    *dist = length(pt - c);
    OPS(6 + 4 + 6);
    *cp = c;
    *t = tt;
}
static void quadratic_closest_pt_approx(V2 p0, V2 p1, V2 p2, V2 pt, V2* cp_out, float* t_out) {
    V2 b0 = p0 - pt, b1 = p1 - pt, b2 = p2 - pt;  // curve.rs:267-296
    float a = cross(b0, b2);
    float b = 2.0f * cross(b1, b0);
    float d = 2.0f * cross(b2, b1);
    float f = b * d - a * a;
    V2 d21 = b2 - b1, d10 = b1 - b0, d20 = b2 - b0;
    V2 gf = (d21 * b) + (d10 * d) + (d20 * a);
    gf = gf * 2.0f;
    gf = mk(gf.y, -gf.x);
    float t = 0.0f;
    float denom = dot(gf, gf);
    OPS(6 + 3 + 4 + 4 + 3 + 6 + 10 + 2 + 3);
    if (denom > 1.0e-8f) {
        V2 pp = gf * (-f / denom);
        V2 d0p = b0 - pp;
        float ap = cross(d0p, d20);
        float bp = 2.0f * cross(d10, d0p);
        float denom2 = 2.0f * a + b + d;
        OPS(3 + 2 + 3 + 4 + 3);
        if (std::fabs(denom2) > 1.0e-8f) t = (OPS(2), clampf((ap + bp) / denom2, 0.0f, 1.0f));
    }
    float tt = 1.0f - t;
    *cp_out = p0 * (tt * tt) + p1 * (2.0f * tt * t) + p2 * (t * t);
    OPS(1 + 14);
    *t_out = t;
}
static CP closest_point_quadratic(V2 pt, V2 p0, V2 p1, V2 p2, bool approx) {  // curve.rs:26-78
    if (approx) {
        V2 cp;
        float t;
        quadratic_closest_pt_approx(p0, p1, p2, pt, &cp, &t);
        OPS(6);
        return CP{cp, t, length(pt - cp)};
    }
    float best_t = 0.0f;
    V2 best_pt = p0;
    float best_dist = length(pt - p0);
    float dist_end = length(pt - p2);
    if (dist_end < best_dist) {
        best_dist = dist_end;
        best_pt = p2;
        best_t = 1.0f;
    }
    double ax = (double)(p0.x - 2.0f * p1.x + p2.x);
    double ay = (double)(p0.y - 2.0f * p1.y + p2.y);
    double bx = (double)(-p0.x + p1.x);
    double by = (double)(-p0.y + p1.y);
    double cx = (double)(p0.x - pt.x);
    double cy = (double)(p0.y - pt.y);
    double a = ax * ax + ay * ay;
    double b = 3.0 * (ax * bx + ay * by);
    double c = 2.0 * (bx * bx + by * by) + (ax * cx + ay * cy);
    double d = bx * cx + by * cy;
    OPS(12 + 10 + 18);  // end-point distances, coefficients, the cubic's coefficients
    double roots[3] = {0, 0, 0};
    int num = solve_cubic(a, b, c, d, roots);
    for (int i = 0; i < num; ++i) {
        double t = roots[i];
        if (t >= 0.0 && t <= 1.0) {
            float t32 = (float)t;
            float tt = 1.0f - t32;
            V2 cp = (p0 * (tt * tt)) + (p1 * (2.0f * tt * t32)) + (p2 * (t32 * t32));
            float dist = length(pt - cp);
            OPS(1 + 14 + 6);
            if (dist < best_dist) {
                best_dist = dist;
                best_pt = cp;
                best_t = t32;
            }
        }
    }
    return CP{best_pt, best_t, best_dist};
}
static CP closest_point_cubic_approx(V2 pt, V2 p0, V2 p1, V2 p2, V2 p3) {  // curve.rs:81-119
    const int steps = 8;
    float inv = 1.0f / (float)steps;
    V2 prev = p0;
    float prev_t = 0.0f;
    V2 best_pt = p0;
    float best_t = 0.0f;
    float best_dist = length(pt - p0);
    OPS(6);
    for (int i = 1; i <= steps; ++i) {
        float t = (float)i * inv;
        float tt = 1.0f - t;
        float tt2 = tt * tt, t2 = t * t;
        float a = tt2 * tt, b = 3.0f * tt2 * t, c = 3.0f * tt * t2, d = t2 * t;
        V2 curr = mk(a * p0.x + b * p1.x + c * p2.x + d * p3.x, a * p0.y + b * p1.y + c * p2.y + d * p3.y);
        float dist, seg_t;
        V2 cp;
        distance_to_segment(pt, prev, curr, &dist, &cp, &seg_t);
        float local_t = prev_t + seg_t * (t - prev_t);
        OPS(10 + 14 + 3);
        if (dist < best_dist) {
            best_dist = dist;
            best_pt = cp;
            best_t = local_t;
        }
        prev = curr;
        prev_t = t;
    }
    return CP{best_pt, best_t, best_dist};
}
static CP closest_point_cubic(V2 pt, V2 p0, V2 p1, V2 p2, V2 p3, bool approx) {  // curve.rs:124-264
    if (approx) return closest_point_cubic_approx(pt, p0, p1, p2, p3);
    float best_t = 0.0f;
    V2 best_pt = p0;
    float best_dist = length(pt - p0);
    float dist_end = length(pt - p3);
    if (dist_end < best_dist) {
        best_dist = dist_end;
        best_pt = p3;
        best_t = 1.0f;
    }
    double ax = (double)(-p0.x + 3.0f * p1.x - 3.0f * p2.x + p3.x);
    double ay = (double)(-p0.y + 3.0f * p1.y - 3.0f * p2.y + p3.y);
    double bx = (double)(3.0f * p0.x - 6.0f * p1.x + 3.0f * p2.x);
    double by = (double)(3.0f * p0.y - 6.0f * p1.y + 3.0f * p2.y);
    double cx = (double)(-3.0f * p0.x + 3.0f * p1.x);
    double cy = (double)(-3.0f * p0.y + 3.0f * p1.y);
    double dx = (double)(p0.x - pt.x);
    double dy = (double)(p0.y - pt.y);
    double a = 3.0 * (ax * ax + ay * ay);
    OPS(12 + 28 + 4);  // end-point distances, coefficients, leading term
    if (std::fabs(a) < 1.0e-10) return CP{best_pt, best_t, best_dist};
    OPS(32 + 5 + 16);  // b..f, their normalisation, the deflated cubic and -b/5
    double b = 5.0 * (ax * bx + ay * by);
    double c = 4.0 * (ax * cx + ay * cy) + 2.0 * (bx * bx + by * by);
    double d = 3.0 * ((bx * cx + by * cy) + (ax * dx + ay * dy));
    double e = (cx * cx + cy * cy) + 2.0 * (dx * bx + dy * by);
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
    double p_roots[3] = {0, 0, 0};
    int num_p = solve_cubic(p1a, p1b, p1c, p1d, p_roots);
    double intervals[4] = {0, 0, 0, 0};
    int num_intervals = 0;
    if (q_root >= 0.0 && q_root <= 1.0) intervals[num_intervals++] = q_root;
    for (int i = 0; i < num_p; ++i) intervals[num_intervals++] = p_roots[i];
    for (int j = 1; j < num_intervals; ++j) {
        int k = j;
        while (k > 0 && intervals[k - 1] > intervals[k]) {
            std::swap(intervals[k - 1], intervals[k]);
            k -= 1;
        }
    }
    auto eval_poly = [&](double t) { return ((((t + b) * t + c) * t + d) * t + e) * t + f; };
    auto eval_deriv = [&](double t) {
        return (((5.0 * t + 4.0 * b) * t + 3.0 * c) * t + 2.0 * d) * t + e;
    };
    double lower = 0.0;
    for (int j = 0; j <= num_intervals; ++j) {
        if (j < num_intervals && intervals[j] < 0.0) continue;
        double upper = (j < num_intervals) ? std::fmin(intervals[j], 1.0) : 1.0;
        double lb = lower, ub = upper;
        double lb_eval = eval_poly(lb), ub_eval = eval_poly(ub);
        OPS(19);
        if (lb_eval * ub_eval > 0.0) {
            lower = upper;
            continue;
        }
        if (lb_eval > ub_eval) {
            std::swap(lb, ub);
            std::swap(lb_eval, ub_eval);
        }
        double t = 0.5 * (lb + ub);
        OPS(2);
        for (int it = 0; it < 20; ++it) {
            if (!(t >= lb && t <= ub)) t = (OPS(2), 0.5 * (lb + ub));
            double value = eval_poly(t);
            OPS(9);
            if (std::fabs(value) < 1.0e-5 || it == 19) break;
            if (value > 0.0)
                ub = t;
            else
                lb = t;
            double derivative = eval_deriv(t);
            t -= value / derivative;
            OPS(11 + 2);
        }
        if (t >= 0.0 && t <= 1.0) {
            float t32 = (float)t;
            float tt = 1.0f - t32;
            V2 cp = (p0 * (tt * tt * tt)) + (p1 * (3.0f * tt * tt * t32)) +
                    (p2 * (3.0f * tt * t32 * t32)) + (p3 * (t32 * t32 * t32));
            float dist = length(pt - cp);
            OPS(25 + 6);
            if (dist < best_dist) {
                best_dist = dist;
                best_pt = cp;
                best_t = t32;
            }
        }
        if (upper >= 1.0) break;
        lower = upper;
    }
    return CP{best_pt, best_t, best_dist};
}

// ---------------------------------------------------------------- winding (distance/winding.rs:118-192)
static int winding_number_segment(uint8_t kind, V2 p0, V2 p1, V2 p2, V2 p3, V2 pt) {
    if (kind == 0) {
        float dy = p1.y - p0.y;
        OPS(1);
        if (std::fabs(dy) <= 1.0e-8f) return 0;
        float t = (pt.y - p0.y) / dy;
        OPS(2);
        if (t >= 0.0f && t <= 1.0f) {
            float tp = p0.x - pt.x + t * (p1.x - p0.x);
            OPS(4);
            if (tp >= 0.0f) return dy > 0.0f ? 1 : -1;
        }
        return 0;
    }
    if (kind == 1) {
        double a = (double)(p0.y - 2.0f * p1.y + p2.y);
        double b = (double)(-2.0f * p0.y + 2.0f * p1.y);
        double c = (double)(p0.y - pt.y);
        OPS(7);
        double roots[2] = {0, 0};
        int num_roots = 0;
        if (std::fabs(a) < 1.0e-12) {
            if (std::fabs(b) > 1.0e-12) {
                roots[0] = -c / b;
                OPS(1);
                num_roots = 1;
            }
        } else if (solve_quadratic(a, b, c, roots)) {
            num_roots = 2;
        }
        int winding = 0;
        double ax = (double)(p0.x - 2.0f * p1.x + p2.x);
        double bx = (double)(-2.0f * p0.x + 2.0f * p1.x);
        double cx = (double)(p0.x - pt.x);
        OPS(7);
        for (int i = 0; i < num_roots; ++i) {
            double t = roots[i];
            if (t >= 0.0 && t <= 1.0) {
                double tp = ax * t * t + bx * t + cx;
                OPS(5);
                if (tp > 0.0) {
                    double deriv = 2.0 * a * t + b;
                    OPS(3);
                    winding += deriv > 0.0 ? 1 : -1;
                }
            }
        }
        return winding;
    }
    if (kind == 2) {
        double a = (double)(-p0.y + 3.0f * p1.y - 3.0f * p2.y + p3.y);
        double b = (double)(3.0f * p0.y - 6.0f * p1.y + 3.0f * p2.y);
        double c = (double)(-3.0f * p0.y + 3.0f * p1.y);
        double d = (double)(p0.y - pt.y);
        OPS(14);
        double roots[3] = {0, 0, 0};
        int num_roots = solve_cubic(a, b, c, d, roots);
        double ax = (double)(-p0.x + 3.0f * p1.x - 3.0f * p2.x + p3.x);
        double bx = (double)(3.0f * p0.x - 6.0f * p1.x + 3.0f * p2.x);
        double cx = (double)(-3.0f * p0.x + 3.0f * p1.x);
        double dx = (double)(p0.x - pt.x);
        OPS(14);
        int winding = 0;
        for (int i = 0; i < num_roots; ++i) {
            double t = roots[i];
            if (t >= 0.0 && t <= 1.0) {
                double tp = ax * t * t * t + bx * t * t + cx * t + dx;
                OPS(9);
                if (tp > 0.0) {
                    double deriv = 3.0 * a * t * t + 2.0 * b * t + c;
                    OPS(7);
                    winding += deriv > 0.0 ? 1 : -1;
                }
            }
        }
        return winding;
    }
    return 0;
}
static int winding_number_path(const PathG& p, V2 pt) {  // winding.rs:52-70
    if (p.pts.empty()) return 0;
    int winding = 0;
    size_t point_id = 0;
    for (uint8_t nc : p.ncp) {
        V2 q[4];
        size_t next;
        if (!path_segment_points(p, point_id, nc, q, &next)) break;
        winding += winding_number_segment(nc, q[0], q[1], q[2], q[3], pt);
        point_id = next;
    }
    return winding;
}

// ---------------------------------------------------------------- shapes (distance/shape.rs)
struct Bounds {  // distance/bvh.rs:70-114
    V2 min, max;
    static Bounds empty() { return Bounds{mk(INF_F, INF_F), mk(-INF_F, -INF_F)}; }
    void include(const Bounds& o) {
        min = vmin(min, o.min);
        max = vmax(max, o.max);
    }
    V2 center() const { return (min + max) * 0.5f; }
    V2 extent() const { return max - min; }
    bool contains(V2 p) const { return p.x >= min.x && p.x <= max.x && p.y >= min.y && p.y <= max.y; }
    float distance(V2 p) const {
        float dx = std::fmax(std::fmax(min.x - p.x, 0.0f), p.x - max.x);
        float dy = std::fmax(std::fmax(min.y - p.y, 0.0f), p.y - max.y);
        return std::sqrt(dx * dx + dy * dy);
    }
};
static Bounds bounds_from_points(const std::vector<V2>& pts) {  // path_utils.rs:107-115
    Bounds b = Bounds::empty();
    for (V2 p : pts) {
        b.min = vmin(b.min, p);
        b.max = vmax(b.max, p);
    }
    return b;
}
static Bounds inflate_bounds(Bounds b, float pad) {  // shape.rs:92-99
    pad = std::fmax(pad, 0.0f);
    return Bounds{mk(b.min.x - pad, b.min.y - pad), mk(b.max.x + pad, b.max.y + pad)};
}
static V2 ellipse_extents(const M3& t, float rx, float ry) {  // shape.rs:81-89
    float m00 = t.m[0][0], m01 = t.m[0][1], m10 = t.m[1][0], m11 = t.m[1][1];
    float ex = std::sqrt((m00 * rx) * (m00 * rx) + (m01 * ry) * (m01 * ry));
    float ey = std::sqrt((m10 * rx) * (m10 * rx) + (m11 * ry) * (m11 * ry));
    return mk(ex, ey);
}
static bool shape_geom_bounds(const Shape& s, Bounds* out) {  // shape.rs:17-59
    const M3& t = s.transform;
    if (s.kind == DVG_SHAPE_CIRCLE || s.kind == DVG_SHAPE_ELLIPSE) {
        V2 c = xform_pt(t, mk(s.prm[0], s.prm[1]));
        float rx = std::fabs(s.prm[2]);
        float ry = s.kind == DVG_SHAPE_CIRCLE ? rx : std::fabs(s.prm[3]);
        V2 ext = ellipse_extents(t, rx, ry);
        *out = Bounds{mk(c.x - ext.x, c.y - ext.y), mk(c.x + ext.x, c.y + ext.y)};
        return true;
    }
    if (s.kind == DVG_SHAPE_RECT) {
        std::vector<V2> corners = {xform_pt(t, mk(s.prm[0], s.prm[1])), xform_pt(t, mk(s.prm[2], s.prm[1])),
                                   xform_pt(t, mk(s.prm[2], s.prm[3])), xform_pt(t, mk(s.prm[0], s.prm[3]))};
        *out = bounds_from_points(corners);
        return true;
    }
    if (s.kind == DVG_SHAPE_PATH) {
        if (s.path.pts.empty()) return false;
        std::vector<V2> pts = s.path.pts;
        if (!is_identity(t))  // path_utils.rs:88-104
            for (auto& p : pts) p = xform_pt(t, p);
        *out = bounds_from_points(pts);
        return true;
    }
    return false;
}
static float max_stroke_radius(const Shape& s) {  // shape.rs:62-78
    float stroke_scale = std::fmax(max_scale(s.transform), 0.0f);
    float radius = std::fabs(s.stroke_width) * stroke_scale;
    if (s.kind == DVG_SHAPE_PATH && s.path.has_thick) {
        float mt = 0.0f;
        for (float v : s.path.thick) mt = std::fmax(mt, std::fabs(v));
        radius = std::fmax(radius, mt * stroke_scale);
    }
    float pm = s.join == DVG_JOIN_MITER ? std::fmax(s.miter, 1.0f) : 1.0f;
    // extension: square caps reach sqrt(2) (rounded up) radii from an open path's ends
    if (s.kind == DVG_SHAPE_PATH && !s.path.closed && s.cap == DVG_CAP_SQUARE) pm = std::fmax(pm, 1.41422f);
    if (radius > 0.0f) radius *= pm;
    return radius;
}
static bool shape_bounds(const Shape& s, Bounds* out) {  // shape.rs:9-14
    Bounds g;
    if (!shape_geom_bounds(s, &g)) return false;
    *out = inflate_bounds(g, max_stroke_radius(s));
    return true;
}
static V2 closest_point_circle(V2 c, float r, V2 pt) {  // shape.rs:106-113
    V2 d = pt - c;
    float len = length(d);
    if (len <= 1.0e-8f) return mk(c.x + r, c.y);
    return c + d * (r / len);
}
static V2 closest_point_ellipse(V2 c, V2 radius, V2 pt) {  // shape.rs:116-164
    float rx = std::fabs(radius.x), ry = std::fabs(radius.y);
    const float eps = 1.0e-6f;
    if (rx < eps && ry < eps) return c;
    if (rx < eps) return mk(c.x, c.y + clampf(pt.y - c.y, -ry, ry));
    if (ry < eps) return mk(c.x + clampf(pt.x - c.x, -rx, rx), c.y);
    float dx = pt.x - c.x, dy = pt.y - c.y;
    if (std::fabs(dx) < eps && std::fabs(dy) < eps) return mk(c.x + rx, c.y);
    float sign_x = dx < 0.0f ? -1.0f : 1.0f;
    float sign_y = dy < 0.0f ? -1.0f : 1.0f;
    dx = std::fabs(dx);
    dy = std::fabs(dy);
    float t = std::atan2(dy * rx, dx * ry);
    OPS(2 + 3);
    const int max_iter = 20;
    const float tol = 1.0e-6f;
    for (int i = 0; i < max_iter; ++i) {
        float s = std::sin(t), co = std::cos(t);
        float g = rx * dx * s - ry * dy * co + (ry * ry - rx * rx) * s * co;
        float g_t = rx * dx * co + ry * dy * s + (ry * ry - rx * rx) * (co * co - s * s);
        OPS(2 + 11 + 12);
        if (std::fabs(g_t) < 1.0e-12f) break;
        float next = clampf(t - g / g_t, 0.0f, FRAC_PI_2_F);
        OPS(3);
        if (std::fabs(next - t) < tol) {
            t = next;
            break;
        }
        t = next;
    }
    float s = std::sin(t), co = std::cos(t);
    OPS(2 + 6);
    return mk(c.x + sign_x * rx * co, c.y + sign_y * ry * s);
}
static V2 closest_point_rect(V2 mn, V2 mx, V2 pt) {  // shape.rs:167-185
    bool inside = pt.x >= mn.x && pt.x <= mx.x && pt.y >= mn.y && pt.y <= mx.y;
    if (!inside) return mk(clampf(pt.x, mn.x, mx.x), clampf(pt.y, mn.y, mx.y));
    float dl = pt.x - mn.x, dr = mx.x - pt.x, db = pt.y - mn.y, dt = mx.y - pt.y;
    if (dl <= dr && dl <= db && dl <= dt) return mk(mn.x, pt.y);
    if (dr <= db && dr <= dt) return mk(mx.x, pt.y);
    if (db <= dt) return mk(pt.x, mn.y);
    return mk(pt.x, mx.y);
}
static float rect_signed_distance(V2 pt, V2 mn, V2 mx) {  // shape.rs:188-201
    float dx = std::fmax(std::fmax(mn.x - pt.x, 0.0f), pt.x - mx.x);
    float dy = std::fmax(std::fmax(mn.y - pt.y, 0.0f), pt.y - mx.y);
    float outside = std::sqrt(dx * dx + dy * dy);
    float inside = std::fmin(std::fmin(std::fmin(pt.x - mn.x, mx.x - pt.x), pt.y - mn.y), mx.y - pt.y);
    OPS(4 + 4 + 4);
    return outside > 0.0f ? outside : -inside;
}
static float ellipse_signed_distance(V2 pt, V2 c, V2 radius) {  // shape.rs:204-212
    float rx = std::fmax(std::fabs(radius.x), 1.0e-6f);
    float ry = std::fmax(std::fabs(radius.y), 1.0e-6f);
    V2 local = pt - c;
    bool inside = (local.x / rx) * (local.x / rx) + (local.y / ry) * (local.y / ry) <= 1.0f;
    V2 closest = closest_point_ellipse(c, mk(rx, ry), pt);
    float dist = length(pt - closest);
    OPS(2 + 7 + 6);
    return inside ? -dist : dist;
}

// ---------------------------------------------------------------- BVH (distance/bvh.rs)
static const uint32_t BVH_NONE = 0xffffffffu;
static const size_t BVH_LEAF_SIZE = 8;
struct BvhNode {
    Bounds bounds;
    uint32_t left, right, start, count;
};
struct SegData {  // bvh.rs:130-154
    size_t segment_index;
    uint8_t kind;
    V2 p0, p1, p2, p3;
    float r0, r1, r2, r3;
    Bounds bounds;
};
struct PathBvh {
    std::vector<BvhNode> nodes;
    std::vector<size_t> indices;
    std::vector<SegData> segments;
    bool approx = false;
};
struct BvhShape {
    size_t shape_index;
    Bounds bounds;
    bool has_path_bvh = false;
    PathBvh path_bvh;
};
struct GroupBvh {
    std::vector<BvhNode> nodes;
    std::vector<size_t> indices;
    std::vector<BvhShape> shapes;
};
struct SceneBvh {
    std::vector<GroupBvh> groups;
};

template <typename BoundsOf>
static uint32_t build_node(std::vector<BvhNode>& nodes, BoundsOf bounds_of, std::vector<size_t>& idx,
                           size_t start, size_t end) {  // bvh.rs:190-238 / 384-432
    Bounds b = Bounds::empty();
    for (size_t i = start; i < end; ++i) b.include(bounds_of(idx[i]));
    size_t count = end - start;
    uint32_t node_index = (uint32_t)nodes.size();
    nodes.push_back(BvhNode{b, BVH_NONE, BVH_NONE, (uint32_t)start, (uint32_t)count});
    if (count <= BVH_LEAF_SIZE) return node_index;
    V2 ext = b.extent();
    int axis = ext.x >= ext.y ? 0 : 1;
    std::stable_sort(idx.begin() + start, idx.begin() + end, [&](size_t a, size_t c) {
        V2 ca = bounds_of(a).center(), cb = bounds_of(c).center();
        float va = axis == 0 ? ca.x : ca.y, vb = axis == 0 ? cb.x : cb.y;
        return va < vb;
    });
    size_t mid = start + count / 2;
    uint32_t l = build_node(nodes, bounds_of, idx, start, mid);
    uint32_t r = build_node(nodes, bounds_of, idx, mid, end);
    nodes[node_index].left = l;
    nodes[node_index].right = r;
    nodes[node_index].count = 0;
    return node_index;
}
static Bounds segment_bounds(std::initializer_list<V2> pts, float pad) {  // shape.rs:102-105
    Bounds b = Bounds::empty();
    for (V2 p : pts) {
        b.min = vmin(b.min, p);
        b.max = vmax(b.max, p);
    }
    return inflate_bounds(b, pad);
}
// The path's segments in path order with per-point radii (bvh.rs:255-364).
static std::vector<SegData> path_segments(const Shape& s, float dr) {
    const PathG& p = s.path;
    size_t point_id = 0;
    std::vector<SegData> segs;
    if (p.pts.empty()) return segs;
    for (size_t si = 0; si < p.ncp.size(); ++si) {
        uint8_t nc = p.ncp[si];
        V2 q[4];
        float r[4];
        if (nc == 0) {
            if (!path_point_radius(p, point_id, dr, &q[0], &r[0])) break;
            if (!path_point_radius(p, point_id + 1, dr, &q[1], &r[1])) break;
            segs.push_back(SegData{si, 0, q[0], q[1], q[1], q[1], r[0], r[1], r[1], r[1],
                                   segment_bounds({q[0], q[1]}, std::fmax(r[0], r[1]))});
            point_id += 1;
        } else if (nc == 1) {
            if (!path_point_radius(p, point_id, dr, &q[0], &r[0])) break;
            if (!path_point_radius(p, point_id + 1, dr, &q[1], &r[1])) break;
            if (!path_point_radius(p, point_id + 2, dr, &q[2], &r[2])) break;
            segs.push_back(SegData{si, 1, q[0], q[1], q[2], q[2], r[0], r[1], r[2], r[2],
                                   segment_bounds({q[0], q[1], q[2]}, std::fmax(std::fmax(r[0], r[1]), r[2]))});
            point_id += 2;
        } else if (nc == 2) {
            if (!path_point_radius(p, point_id, dr, &q[0], &r[0])) break;
            if (!path_point_radius(p, point_id + 1, dr, &q[1], &r[1])) break;
            if (!path_point_radius(p, point_id + 2, dr, &q[2], &r[2])) break;
            if (!path_point_radius(p, point_id + 3, dr, &q[3], &r[3])) break;
            segs.push_back(SegData{si, 2, q[0], q[1], q[2], q[3], r[0], r[1], r[2], r[3],
                                   segment_bounds({q[0], q[1], q[2], q[3]},
                                                  std::fmax(std::fmax(std::fmax(r[0], r[1]), r[2]), r[3]))});
            point_id += 3;
        } else {
            break;
        }
    }
    return segs;
}
static bool build_path_bvh(const Shape& s, PathBvh* out) {  // bvh.rs:241-381
    if (s.kind != DVG_SHAPE_PATH) return false;
    if (s.path.pts.empty()) return false;
    std::vector<SegData> segs = path_segments(s, s.stroke_width);
    if (segs.empty()) return false;
    out->segments = segs;
    out->indices.resize(segs.size());
    for (size_t i = 0; i < segs.size(); ++i) out->indices[i] = i;
    out->nodes.clear();
    build_node(out->nodes, [&](size_t i) { return out->segments[i].bounds; }, out->indices, 0, segs.size());
    out->approx = s.path.approx;
    return true;
}
static GroupBvh build_group_bvh(const Scene& sc, const Group& g) {  // bvh.rs:156-187
    GroupBvh gb;
    for (size_t si : g.shape_ids) {
        if (si >= sc.shapes.size()) continue;
        const Shape& s = sc.shapes[si];
        Bounds b;
        if (shape_bounds(s, &b)) {
            BvhShape bs;
            bs.shape_index = si;
            bs.bounds = b;
            bs.has_path_bvh = build_path_bvh(s, &bs.path_bvh);
            gb.shapes.push_back(bs);
        }
    }
    gb.indices.resize(gb.shapes.size());
    for (size_t i = 0; i < gb.shapes.size(); ++i) gb.indices[i] = i;
    if (!gb.indices.empty())
        build_node(gb.nodes, [&](size_t i) { return gb.shapes[i].bounds; }, gb.indices, 0, gb.indices.size());
    return gb;
}
static SceneBvh build_scene_bvh(const Scene& sc) {  // bvh.rs:21-30
    SceneBvh b;
    for (const Group& g : sc.groups) b.groups.push_back(build_group_bvh(sc, g));
    return b;
}

// ---------------------------------------------------------------- closest / within (distance/closest.rs)
static float seg_radius(const SegData& s, float t) {  // closest.rs:66-79
    if (s.kind == 0) return OPS(3), s.r0 + t * (s.r1 - s.r0);
    float tt = 1.0f - t;
    if (s.kind == 1) return OPS(10), tt * tt * s.r0 + 2.0f * tt * t * s.r1 + t * t * s.r2;
    return OPS(18), tt * tt * tt * s.r0 + 3.0f * tt * tt * t * s.r1 + 3.0f * tt * t * t * s.r2 + t * t * t * s.r3;
}
static CP seg_closest(const SegData& s, V2 pt, bool approx) {
    if (s.kind == 0) {
        CP r;
        distance_to_segment(pt, s.p0, s.p1, &r.dist, &r.cp, &r.t);
        return r;
    }
    if (s.kind == 1) return closest_point_quadratic(pt, s.p0, s.p1, s.p2, approx);
    return closest_point_cubic(pt, s.p0, s.p1, s.p2, s.p3, approx);
}
// ---------------------------------------------------------------- stroke joins and caps
// Not in the crate, which strokes every path with round joins and caps (its join and
// cap fields only pad bounds, prepare.rs:207-210): the library's extension, restated
// with the same arithmetic as its kernels.  A path whose join (or, open, cap) is not
// round keeps the crate's segment-body test except that a closest point exactly at
// a segment end with such a join or cap does not count; the join or cap region is
// added instead (bevel triangle; miter quad up to the miter limit, else bevel; butt:
// nothing; square: a rectangle one radius long and two wide beyond the end).
static bool style_nonround(const Shape& s) {
    if (s.kind != DVG_SHAPE_PATH) return false;
    return s.join != DVG_JOIN_ROUND || (!s.path.closed && s.cap != DVG_CAP_ROUND);
}
static bool end_excluded(const Shape& s, size_t seg, size_t nseg, float t) {
    const bool at0 = t == 0.0f, at1 = t == 1.0f;
    if (!style_nonround(s) || !(at0 || at1)) return false;
    const bool join = s.path.closed || (at0 ? seg > 0 : seg + 1 < nseg);
    return join ? s.join != DVG_JOIN_ROUND : s.cap != DVG_CAP_ROUND;
}
static V2 seg_dir0(const SegData& g) {
    V2 d = g.p1 - g.p0;
    if (d.x == 0.0f && d.y == 0.0f) d = g.p2 - g.p0;
    if (d.x == 0.0f && d.y == 0.0f) d = g.p3 - g.p0;
    return d;
}
static V2 seg_dir1(const SegData& g) {
    V2 d = g.p3 - g.p2;
    if (d.x == 0.0f && d.y == 0.0f) d = g.p3 - g.p1;
    if (d.x == 0.0f && d.y == 0.0f) d = g.p3 - g.p0;
    return d;
}
static float cross2f(float ax, float ay, float bx, float by) { return ax * by - ay * bx; }
static bool in_triangle(V2 p, V2 a, V2 b, V2 c) {
    const float d1 = cross2f(b.x - a.x, b.y - a.y, p.x - a.x, p.y - a.y);
    const float d2 = cross2f(c.x - b.x, c.y - b.y, p.x - b.x, p.y - b.y);
    const float d3 = cross2f(a.x - c.x, a.y - c.y, p.x - c.x, p.y - c.y);
    const bool neg = d1 < 0.0f || d2 < 0.0f || d3 < 0.0f, pos = d1 > 0.0f || d2 > 0.0f || d3 > 0.0f;
    return !(neg && pos);
}
static bool join_hit(V2 p, V2 v, V2 din, V2 dout, float r, uint32_t join, float limit) {
    const float li = std::sqrt(din.x * din.x + din.y * din.y), lo = std::sqrt(dout.x * dout.x + dout.y * dout.y);
    if (!(li > 0.0f) || !(lo > 0.0f) || !(r > 0.0f)) return false;
    din = mk(din.x / li, din.y / li);
    dout = mk(dout.x / lo, dout.y / lo);
    const float cr = cross2f(din.x, din.y, dout.x, dout.y);
    if (std::fabs(cr) < 1.0e-6f) return false;
    const float sg = cr > 0.0f ? 1.0f : -1.0f;
    const V2 a = mk(v.x + r * sg * din.y, v.y - r * sg * din.x);
    const V2 b = mk(v.x + r * sg * dout.y, v.y - r * sg * dout.x);
    if (join == DVG_JOIN_MITER) {
        const float sm = cross2f(b.x - a.x, b.y - a.y, dout.x, dout.y) / cr;
        const V2 m = mk(a.x + sm * din.x, a.y + sm * din.y);
        const float ml = std::sqrt((m.x - v.x) * (m.x - v.x) + (m.y - v.y) * (m.y - v.y));
        if (ml <= limit * r) return in_triangle(p, v, a, m) || in_triangle(p, v, m, b);
    }
    return in_triangle(p, v, a, b);
}
static bool square_cap_hit(V2 p, V2 v, V2 d, float r) {
    const float l = std::sqrt(d.x * d.x + d.y * d.y);
    if (!(l > 0.0f) || !(r > 0.0f)) return false;
    const float dx = d.x / l, dy = d.y / l, qx = p.x - v.x, qy = p.y - v.y;
    const float sp = qx * dx + qy * dy, u = qx * -dy + qy * dx;
    return sp >= 0.0f && sp <= r && std::fabs(u) <= r;
}
// segs: the path's segments in path order (quadratics and lines repeat their last point).
static bool join_cap_hit(const Shape& s, const std::vector<SegData>& segs, V2 p) {
    const bool closed = s.path.closed;
    const float limit = std::fmax(s.miter, 1.0f);
    const float reach = (s.join == DVG_JOIN_MITER ? limit : 1.0f) * 1.001f;
    const size_t n = segs.size();
    for (size_t k = 0; k < n; ++k) {
        const SegData& g = segs[k];
        const V2 v = g.p0;
        const float r = g.r0;
        if (k > 0 || closed) {
            if (s.join == DVG_JOIN_ROUND) continue;
            const float dx = p.x - v.x, dy = p.y - v.y;
            if (dx * dx + dy * dy > (reach * r) * (reach * r)) continue;
            const SegData& in = segs[k > 0 ? k - 1 : n - 1];
            if (join_hit(p, v, seg_dir1(in), seg_dir0(g), r, s.join, limit)) return true;
        } else if (s.cap == DVG_CAP_SQUARE) {
            const V2 d = seg_dir0(g);
            if (square_cap_hit(p, v, mk(-d.x, -d.y), r)) return true;
        }
    }
    if (!closed && s.cap == DVG_CAP_SQUARE && n > 0)
        if (square_cap_hit(p, segs[n - 1].p3, seg_dir1(segs[n - 1]), segs[n - 1].r3)) return true;
    return false;
}

static bool within_distance_path_bvh(const PathBvh& pb, V2 pt, const Shape* style) {  // closest.rs:20-98
    if (pb.nodes.empty()) return false;
    std::vector<size_t> stack{0};
    while (!stack.empty()) {
        size_t ni = stack.back();
        stack.pop_back();
        const BvhNode& n = pb.nodes[ni];
        if (!n.bounds.contains(pt)) continue;
        if (n.count > 0) {
            for (size_t i = n.start; i < (size_t)n.start + n.count; ++i) {
                const SegData& s = pb.segments[pb.indices[i]];
                CP c = seg_closest(s, pt, pb.approx);
                if (c.dist < seg_radius(s, c.t) &&
                    !(style && end_excluded(*style, pb.indices[i], pb.segments.size(), c.t)))
                    return true;
            }
        } else {
            if (n.left != BVH_NONE) stack.push_back(n.left);
            if (n.right != BVH_NONE) stack.push_back(n.right);
        }
    }
    return style && style_nonround(*style) && join_cap_hit(*style, pb.segments, pt);
}
struct PathHit {
    bool valid = false;
    size_t segment_index = 0;
    float t = 0.0f;
};
static bool closest_point_path_bvh(const PathBvh& pb, V2 pt, V2* best_pt_out, PathHit* hit) {  // closest.rs:104-199
    if (pb.nodes.empty()) return false;
    float best_dist = INF_F;
    V2 best_pt = mk(0, 0);
    size_t best_seg = 0;
    float best_t = 0.0f;
    std::vector<size_t> stack{0};
    while (!stack.empty()) {
        size_t ni = stack.back();
        stack.pop_back();
        const BvhNode& n = pb.nodes[ni];
        if (n.bounds.distance(pt) > best_dist) continue;
        if (n.count > 0) {
            for (size_t i = n.start; i < (size_t)n.start + n.count; ++i) {
                const SegData& s = pb.segments[pb.indices[i]];
                CP c = seg_closest(s, pt, pb.approx);
                if (c.dist < best_dist) {
                    best_dist = c.dist;
                    best_pt = c.cp;
                    best_seg = s.segment_index;
                    best_t = c.t;
                }
            }
        } else {
            float ld = INF_F, rd = INF_F;
            if (n.left != BVH_NONE) ld = pb.nodes[n.left].bounds.distance(pt);
            if (n.right != BVH_NONE) rd = pb.nodes[n.right].bounds.distance(pt);
            if (ld < rd) {
                if (rd <= best_dist) stack.push_back(n.right);
                if (ld <= best_dist) stack.push_back(n.left);
            } else {
                if (ld <= best_dist) stack.push_back(n.left);
                if (rd <= best_dist) stack.push_back(n.right);
            }
        }
    }
    if (!std::isfinite(best_dist)) return false;
    *best_pt_out = best_pt;
    hit->valid = true;
    hit->segment_index = best_seg;
    hit->t = best_t;
    return true;
}
static bool within_distance_shape(const Shape& s, V2 pt, float r) {  // closest.rs:206-379
    if (r <= 0.0f) return false;
    V2 lp = xform_inv_dist(s.transform, pt);
    if (s.kind == DVG_SHAPE_CIRCLE) {
        float dist = length(lp - mk(s.prm[0], s.prm[1])) - std::fabs(s.prm[2]);
        OPS(7);
        return std::fabs(dist) < r;
    }
    if (s.kind == DVG_SHAPE_ELLIPSE) {
        float dist = ellipse_signed_distance(lp, mk(s.prm[0], s.prm[1]), mk(std::fabs(s.prm[2]), std::fabs(s.prm[3])));
        return std::fabs(dist) < r;
    }
    if (s.kind == DVG_SHAPE_RECT) {
        float dist = rect_signed_distance(lp, mk(s.prm[0], s.prm[1]), mk(s.prm[2], s.prm[3]));
        return std::fabs(dist) < r;
    }
    if (s.kind == DVG_SHAPE_PATH && style_nonround(s)) {  // joins / caps other than round (extension)
        std::vector<SegData> segs = path_segments(s, r);
        for (size_t k = 0; k < segs.size(); ++k) {
            CP c = seg_closest(segs[k], lp, s.path.approx);
            if (c.dist < seg_radius(segs[k], c.t) && !end_excluded(s, k, segs.size(), c.t)) return true;
        }
        return join_cap_hit(s, segs, lp);
    }
    if (s.kind == DVG_SHAPE_PATH) {
        const PathG& p = s.path;
        if (p.pts.empty()) return false;
        size_t point_id = 0;
        for (uint8_t nc : p.ncp) {
            V2 q[4];
            float rr[4];
            if (nc == 0) {
                if (!path_point_radius(p, point_id, r, &q[0], &rr[0])) break;
                if (!path_point_radius(p, point_id + 1, r, &q[1], &rr[1])) break;
                float dist, t;
                V2 cp;
                distance_to_segment(lp, q[0], q[1], &dist, &cp, &t);
                float radius = rr[0] + t * (rr[1] - rr[0]);
                if (dist < radius) return true;
                point_id += 1;
            } else if (nc == 1) {
                if (!path_point_radius(p, point_id, r, &q[0], &rr[0])) break;
                if (!path_point_radius(p, point_id + 1, r, &q[1], &rr[1])) break;
                if (!path_point_radius(p, point_id + 2, r, &q[2], &rr[2])) break;
                CP c = closest_point_quadratic(lp, q[0], q[1], q[2], p.approx);
                float t = c.t, tt = 1.0f - t;
                float radius = tt * tt * rr[0] + 2.0f * tt * t * rr[1] + t * t * rr[2];
                if (c.dist < radius) return true;
                point_id += 2;
            } else if (nc == 2) {
                if (!path_point_radius(p, point_id, r, &q[0], &rr[0])) break;
                if (!path_point_radius(p, point_id + 1, r, &q[1], &rr[1])) break;
                if (!path_point_radius(p, point_id + 2, r, &q[2], &rr[2])) break;
                if (!path_point_radius(p, point_id + 3, r, &q[3], &rr[3])) break;
                CP c = closest_point_cubic(lp, q[0], q[1], q[2], q[3], p.approx);
                float t = c.t, tt = 1.0f - t;
                float radius = tt * tt * tt * rr[0] + 3.0f * tt * tt * t * rr[1] + 3.0f * tt * t * t * rr[2] +
                               t * t * t * rr[3];
                if (c.dist < radius) return true;
                point_id += 3;
            } else {
                break;
            }
        }
        return false;
    }
    return false;
}
static bool closest_point_shape(const Shape& s, V2 pt, V2* out, PathHit* hit) {  // closest.rs:386-456
    V2 lp = xform_inv_dist(s.transform, pt);
    hit->valid = false;
    if (s.kind == DVG_SHAPE_CIRCLE) {
        *out = xform_pt(s.transform, closest_point_circle(mk(s.prm[0], s.prm[1]), std::fabs(s.prm[2]), lp));
        return true;
    }
    if (s.kind == DVG_SHAPE_ELLIPSE) {
        *out = xform_pt(s.transform, closest_point_ellipse(mk(s.prm[0], s.prm[1]),
                                                           mk(std::fabs(s.prm[2]), std::fabs(s.prm[3])), lp));
        return true;
    }
    if (s.kind == DVG_SHAPE_RECT) {
        *out = xform_pt(s.transform, closest_point_rect(mk(s.prm[0], s.prm[1]), mk(s.prm[2], s.prm[3]), lp));
        return true;
    }
    if (s.kind == DVG_SHAPE_PATH) {
        const PathG& p = s.path;
        if (p.pts.empty()) return false;
        float best_dist = INF_F;
        V2 best_pt = mk(0, 0);
        size_t best_seg = 0;
        float best_t = 0.0f;
        size_t point_id = 0;
        for (size_t si = 0; si < p.ncp.size(); ++si) {
            uint8_t nc = p.ncp[si];
            V2 q[4];
            size_t next;
            if (!path_segment_points(p, point_id, nc, q, &next)) break;
            CP c;
            if (nc == 0) {
                distance_to_segment(lp, q[0], q[1], &c.dist, &c.cp, &c.t);
            } else if (nc == 1) {
                c = closest_point_quadratic(lp, q[0], q[1], q[2], p.approx);
            } else if (nc == 2) {
                c = closest_point_cubic(lp, q[0], q[1], q[2], q[3], p.approx);
            } else {
                break;
            }
            if (c.dist < best_dist) {
                best_dist = c.dist;
                best_pt = c.cp;
                best_seg = si;
                best_t = c.t;
            }
            point_id = next;
        }
        if (!std::isfinite(best_dist)) return false;
        *out = xform_pt(s.transform, best_pt);
        hit->valid = true;
        hit->segment_index = best_seg;
        hit->t = best_t;
        return true;
    }
    return false;
}
static int winding_number_path_bvh(const PathBvh& pb, V2 pt) {  // winding.rs:73-115
    if (pb.nodes.empty()) return 0;
    int winding = 0;
    std::vector<size_t> stack{0};
    while (!stack.empty()) {
        size_t ni = stack.back();
        stack.pop_back();
        const BvhNode& n = pb.nodes[ni];
        if (pt.y < n.bounds.min.y || pt.y > n.bounds.max.y || pt.x > n.bounds.max.x) continue;
        if (n.count > 0) {
            for (size_t i = n.start; i < (size_t)n.start + n.count; ++i) {
                const SegData& s = pb.segments[pb.indices[i]];
                winding += winding_number_segment(s.kind, s.p0, s.p1, s.p2, s.p3, pt);
            }
        } else {
            if (n.left != BVH_NONE) stack.push_back(n.left);
            if (n.right != BVH_NONE) stack.push_back(n.right);
        }
    }
    return winding;
}
static int winding_number_shape(const Shape& s, const PathBvh* pb, V2 pt) {  // winding.rs:13-48
    if (s.kind == DVG_SHAPE_CIRCLE) {
        float r = std::fabs(s.prm[2]);
        OPS(6);
        return length_sq(pt - mk(s.prm[0], s.prm[1])) < r * r ? 1 : 0;
    }
    if (s.kind == DVG_SHAPE_ELLIPSE) {
        float rx = std::fmax(std::fabs(s.prm[2]), 1.0e-6f);
        float ry = std::fmax(std::fabs(s.prm[3]), 1.0e-6f);
        float dx = (pt.x - s.prm[0]) / rx, dy = (pt.y - s.prm[1]) / ry;
        OPS(7);
        return dx * dx + dy * dy < 1.0f ? 1 : 0;
    }
    if (s.kind == DVG_SHAPE_RECT) {
        return (pt.x > s.prm[0] && pt.x < s.prm[2] && pt.y > s.prm[1] && pt.y < s.prm[3]) ? 1 : 0;
    }
    if (s.kind == DVG_SHAPE_PATH) return pb ? winding_number_path_bvh(*pb, pt) : winding_number_path(s.path, pt);
    return 0;
}

// ---------------------------------------------------------------- distance API (distance/api.rs)
struct ClosestPoint {
    size_t shape_index;
    V2 point;
    float distance;
    PathHit path;
};
static bool within_distance(const Scene& sc, size_t gi, V2 pt) {  // api.rs:15-33
    if (gi >= sc.groups.size()) return false;
    const Group& g = sc.groups[gi];
    V2 lp = xform_pt(g.c2s, pt);
    for (size_t si : g.shape_ids) {
        if (si >= sc.shapes.size()) continue;
        const Shape& s = sc.shapes[si];
        if (s.stroke_width <= 0.0f) continue;
        if (within_distance_shape(s, lp, s.stroke_width)) return true;
    }
    return false;
}
static bool compute_distance(const Scene& sc, size_t gi, V2 pt, float max_radius, ClosestPoint* best) {  // api.rs:36-76
    if (gi >= sc.groups.size()) return false;
    const Group& g = sc.groups[gi];
    V2 lp = xform_pt(g.c2s, pt);
    bool have = false;
    for (size_t si : g.shape_ids) {
        if (si >= sc.shapes.size()) continue;
        V2 lc;
        PathHit ph;
        if (!closest_point_shape(sc.shapes[si], lp, &lc, &ph)) continue;
        V2 closest = xform_pt(g.s2c, lc);
        float distance = length(closest - pt);
        if (distance <= max_radius) {
            if (!have || distance < best->distance) {
                *best = ClosestPoint{si, closest, distance, ph};
                have = true;
            }
        }
    }
    return have;
}
static bool within_distance_bvh(const Scene& sc, const SceneBvh& bvh, size_t gi, V2 pt) {  // api.rs:79-135
    if (gi >= sc.groups.size() || gi >= bvh.groups.size()) return false;
    const Group& g = sc.groups[gi];
    const GroupBvh& gb = bvh.groups[gi];
    if (gb.nodes.empty()) return within_distance(sc, gi, pt);
    V2 lp = xform_pt(g.c2s, pt);
    std::vector<size_t> stack{0};
    while (!stack.empty()) {
        size_t ni = stack.back();
        stack.pop_back();
        const BvhNode& n = gb.nodes[ni];
        if (!n.bounds.contains(lp)) continue;
        if (n.count > 0) {
            for (size_t i = n.start; i < (size_t)n.start + n.count; ++i) {
                const BvhShape& bs = gb.shapes[gb.indices[i]];
                if (bs.shape_index >= sc.shapes.size()) continue;
                const Shape& s = sc.shapes[bs.shape_index];
                if (s.stroke_width <= 0.0f) continue;
                if (bs.has_path_bvh) {
                    V2 sp = xform_inv_dist(s.transform, lp);
                    if (within_distance_path_bvh(bs.path_bvh, sp, &s)) return true;
                } else if (within_distance_shape(s, lp, s.stroke_width)) {
                    return true;
                }
            }
        } else {
            if (n.left != BVH_NONE) stack.push_back(n.left);
            if (n.right != BVH_NONE) stack.push_back(n.right);
        }
    }
    return false;
}
static bool compute_distance_bvh(const Scene& sc, const SceneBvh& bvh, size_t gi, V2 pt, float max_radius,
                                 ClosestPoint* best) {  // api.rs:138-236
    if (gi >= sc.groups.size() || gi >= bvh.groups.size()) return false;
    const Group& g = sc.groups[gi];
    const GroupBvh& gb = bvh.groups[gi];
    if (gb.nodes.empty()) return compute_distance(sc, gi, pt, max_radius, best);
    V2 lp = xform_pt(g.c2s, pt);
    bool have = false;
    float best_dist = max_radius;
    std::vector<size_t> stack{0};
    while (!stack.empty()) {
        size_t ni = stack.back();
        stack.pop_back();
        const BvhNode& n = gb.nodes[ni];
        if (n.bounds.distance(lp) > best_dist) continue;
        if (n.count > 0) {
            for (size_t i = n.start; i < (size_t)n.start + n.count; ++i) {
                const BvhShape& bs = gb.shapes[gb.indices[i]];
                if (bs.shape_index >= sc.shapes.size()) continue;
                const Shape& s = sc.shapes[bs.shape_index];
                V2 lc;
                PathHit ph;
                bool ok;
                if (bs.has_path_bvh) {
                    V2 sp = xform_inv_dist(s.transform, lp);
                    V2 sc_pt;
                    ok = closest_point_path_bvh(bs.path_bvh, sp, &sc_pt, &ph);
                    if (ok) lc = xform_pt(s.transform, sc_pt);
                } else {
                    ok = closest_point_shape(s, lp, &lc, &ph);
                }
                if (!ok) continue;
                V2 closest = xform_pt(g.s2c, lc);
                float distance = length(closest - pt);
                if (distance <= best_dist) {
                    best_dist = distance;
                    *best = ClosestPoint{bs.shape_index, closest, distance, ph};
                    have = true;
                }
            }
        } else {
            float ld = INF_F, rd = INF_F;
            if (n.left != BVH_NONE) ld = gb.nodes[n.left].bounds.distance(lp);
            if (n.right != BVH_NONE) rd = gb.nodes[n.right].bounds.distance(lp);
            if (ld < rd) {
                if (rd <= best_dist) stack.push_back(n.right);
                if (ld <= best_dist) stack.push_back(n.left);
            } else {
                if (ld <= best_dist) stack.push_back(n.left);
                if (rd <= best_dist) stack.push_back(n.right);
            }
        }
    }
    return have;
}
static bool fill_rule_hit(uint32_t rule, int winding) {
    if (rule == DVG_FILL_EVENODD) return (std::abs(winding) % 2) == 1;
    return winding != 0;
}
static bool is_inside(const Scene& sc, size_t gi, V2 pt) {  // api.rs:239-256
    if (gi >= sc.groups.size()) return false;
    const Group& g = sc.groups[gi];
    V2 lp = xform_pt(g.c2s, pt);
    int winding = 0;
    for (size_t si : g.shape_ids) {
        if (si >= sc.shapes.size()) continue;
        const Shape& s = sc.shapes[si];
        winding += winding_number_shape(s, nullptr, xform_inv_dist(s.transform, lp));
    }
    return fill_rule_hit(g.fill_rule, winding);
}
static bool is_inside_bvh(const Scene& sc, const SceneBvh& bvh, size_t gi, V2 pt) {  // api.rs:259-309
    if (gi >= sc.groups.size() || gi >= bvh.groups.size()) return false;
    const Group& g = sc.groups[gi];
    const GroupBvh& gb = bvh.groups[gi];
    if (gb.nodes.empty()) return is_inside(sc, gi, pt);
    V2 lp = xform_pt(g.c2s, pt);
    if (!gb.nodes[0].bounds.contains(lp)) return false;
    int winding = 0;
    std::vector<size_t> stack{0};
    while (!stack.empty()) {
        size_t ni = stack.back();
        stack.pop_back();
        const BvhNode& n = gb.nodes[ni];
        if (!n.bounds.contains(lp)) continue;
        if (n.count > 0) {
            for (size_t i = n.start; i < (size_t)n.start + n.count; ++i) {
                const BvhShape& bs = gb.shapes[gb.indices[i]];
                if (bs.shape_index >= sc.shapes.size()) continue;
                const Shape& s = sc.shapes[bs.shape_index];
                V2 sp = xform_inv_dist(s.transform, lp);
                winding += winding_number_shape(s, bs.has_path_bvh ? &bs.path_bvh : nullptr, sp);
            }
        } else {
            if (n.left != BVH_NONE) stack.push_back(n.left);
            if (n.right != BVH_NONE) stack.push_back(n.right);
        }
    }
    return fill_rule_hit(g.fill_rule, winding);
}

// ---------------------------------------------------------------- gradients (SceneGrad, src/grad.rs:113-126)
struct Grads {
    std::vector<float> shape_params, shape_transform, stroke_width, points, thickness, group_transform,
        paint_params, stop_offsets, stop_colors, bg_image, translation;
    float filter_radius = 0.0f;
    float background[4] = {0, 0, 0, 0};
    bool has_bg_image = false, has_translation = false;
    void init(const Scene& sc, const dvg_scene_desc* d, bool bg_img, bool trans) {
        shape_params.assign((size_t)4 * sc.shapes.size(), 0.0f);
        shape_transform.assign((size_t)9 * sc.shapes.size(), 0.0f);
        stroke_width.assign(sc.shapes.size(), 0.0f);
        points.assign((size_t)2 * d->total_points, 0.0f);
        thickness.assign(d->total_points, 0.0f);
        group_transform.assign((size_t)9 * sc.groups.size(), 0.0f);
        paint_params.assign((size_t)4 * sc.paints.size(), 0.0f);
        stop_offsets.assign(d->total_stops, 0.0f);
        stop_colors.assign((size_t)4 * d->total_stops, 0.0f);
        has_bg_image = bg_img;
        if (bg_img) bg_image.assign((size_t)sc.w * sc.h * 4, 0.0f);
        has_translation = trans;
        if (trans) translation.assign((size_t)sc.w * sc.h * 2, 0.0f);
    }
    void add(const Grads& o) {
        auto addv = [](std::vector<float>& a, const std::vector<float>& b) {
            for (size_t i = 0; i < a.size() && i < b.size(); ++i) a[i] += b[i];
        };
        addv(shape_params, o.shape_params);
        addv(shape_transform, o.shape_transform);
        addv(stroke_width, o.stroke_width);
        addv(points, o.points);
        addv(thickness, o.thickness);
        addv(group_transform, o.group_transform);
        addv(paint_params, o.paint_params);
        addv(stop_offsets, o.stop_offsets);
        addv(stop_colors, o.stop_colors);
        addv(bg_image, o.bg_image);
        addv(translation, o.translation);
        filter_radius += o.filter_radius;
        for (int i = 0; i < 4; ++i) background[i] += o.background[i];
    }
};

// ---------------------------------------------------------------- backward math (backward/math.rs)
static inline float smoothstep(float d) {  // math.rs:9-12
    float t = clampf((d + 1.0f) * 0.5f, 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
static inline V2 normalize(V2 v) {  // math.rs:43-50
    float len = length(v);
    if (len == 0.0f) return mk(0, 0);
    return v / len;
}
static void d_xform_pt(const M3& m, V2 pt, V2 d_out, M3* d_m, V2* d_pt) {  // math.rs:109-128
    float t0 = m.m[0][0] * pt.x + m.m[0][1] * pt.y + m.m[0][2];
    float t1 = m.m[1][0] * pt.x + m.m[1][1] * pt.y + m.m[1][2];
    float t2 = m.m[2][0] * pt.x + m.m[2][1] * pt.y + m.m[2][2];
    V2 out = mk(t0 / t2, t1 / t2);
    float d_t0 = d_out.x / t2;
    float d_t1 = d_out.y / t2;
    float d_t2 = -(d_out.x * out.x + d_out.y * out.y) / t2;
    d_m->m[0][0] += d_t0 * pt.x;
    d_m->m[0][1] += d_t0 * pt.y;
    d_m->m[0][2] += d_t0;
    d_m->m[1][0] += d_t1 * pt.x;
    d_m->m[1][1] += d_t1 * pt.y;
    d_m->m[1][2] += d_t1;
    d_m->m[2][0] += d_t2 * pt.x;
    d_m->m[2][1] += d_t2 * pt.y;
    d_m->m[2][2] += d_t2;
    d_pt->x += d_t0 * m.m[0][0] + d_t1 * m.m[1][0] + d_t2 * m.m[2][0];
    d_pt->y += d_t0 * m.m[0][1] + d_t1 * m.m[1][1] + d_t2 * m.m[2][1];
}
static V2 xform_normal(const M3& m_inv, V2 n) {  // math.rs:139-143
    float x = m_inv.m[0][0] * n.x + m_inv.m[1][0] * n.y;
    float y = m_inv.m[0][1] * n.x + m_inv.m[1][1] * n.y;
    return normalize(mk(x, y));
}
static M3 transpose3(const M3& m) {
    M3 o;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o.m[r][c] = m.m[c][r];
    return o;
}
static V2 d_length(V2 v, float d_l) {  // math.rs:33-41
    float l_sq = dot(v, v);
    float l = std::sqrt(l_sq);
    if (l == 0.0f) return mk(0, 0);
    float d_l_sq = 0.5f * d_l / l;
    return v * (2.0f * d_l_sq);
}

// ---------------------------------------------------------------- paint (backward/paint.rs)
static V4 stops_color(const Paint& p, float t) {  // paint.rs:16-39 (shared by linear / radial)
    if (p.stops.empty()) return V4{0, 0, 0, 0};
    if (t < p.stops[0].offset) {
        Color c = p.stops[0].color;
        return V4{c.r, c.g, c.b, c.a};
    }
    for (size_t i = 0; i + 1 < p.stops.size(); ++i) {
        const Stop& cu = p.stops[i];
        const Stop& nx = p.stops[i + 1];
        if (t >= cu.offset && t < nx.offset) {
            float tt = (t - cu.offset) / (nx.offset - cu.offset);
            Color c0 = cu.color, c1 = nx.color;
            return V4{c0.r * (1.0f - tt) + c1.r * tt, c0.g * (1.0f - tt) + c1.g * tt,
                      c0.b * (1.0f - tt) + c1.b * tt, c0.a * (1.0f - tt) + c1.a * tt};
        }
    }
    Color l = p.stops.back().color;
    return V4{l.r, l.g, l.b, l.a};
}
static V4 paint_color(const Paint& p, V2 pt) {  // paint.rs:8-74
    if (p.kind == DVG_PAINT_SOLID) return V4{p.p[0], p.p[1], p.p[2], p.p[3]};
    if (p.kind == DVG_PAINT_LINEAR) {
        V2 beg = mk(p.p[0], p.p[1]), end = mk(p.p[2], p.p[3]);
        float denom = std::fmax(dot(end - beg, end - beg), 1.0e-3f);
        float t = dot(pt - beg, end - beg) / denom;
        return stops_color(p, t);
    }
    if (p.kind == DVG_PAINT_RADIAL) {
        V2 off = pt - mk(p.p[0], p.p[1]);
        V2 nrm = mk(off.x / p.p[2], off.y / p.p[3]);
        float t = length(nrm);
        return stops_color(p, t);
    }
    return V4{0, 0, 0, 0};
}
static void add_stop_color(Grads& g, uint32_t stop_base, size_t i, V4 c) {
    float* sc = &g.stop_colors[4 * (stop_base + i)];
    sc[0] += c.x;
    sc[1] += c.y;
    sc[2] += c.z;
    sc[3] += c.w;
}
static void d_sample_paint(const Scene& sc, int pi, Grads& g, V2 pt, V4 d_color, V2* d_translation) {  // paint.rs:77-280
    const Paint& p = sc.paints[pi];
    float* dp = &g.paint_params[4 * (size_t)pi];
    uint32_t sb = sc.paint_stop_base[pi];
    if (p.kind == DVG_PAINT_SOLID) {
        dp[0] += d_color.x;
        dp[1] += d_color.y;
        dp[2] += d_color.z;
        dp[3] += d_color.w;
        return;
    }
    if (p.kind != DVG_PAINT_LINEAR && p.kind != DVG_PAINT_RADIAL) return;
    float t;
    V2 beg, end, off, nrm;
    float denom = 0.0f;
    if (p.kind == DVG_PAINT_LINEAR) {
        beg = mk(p.p[0], p.p[1]);
        end = mk(p.p[2], p.p[3]);
        denom = std::fmax(dot(end - beg, end - beg), 1.0e-3f);
        t = dot(pt - beg, end - beg) / denom;
    } else {
        off = pt - mk(p.p[0], p.p[1]);
        nrm = mk(off.x / p.p[2], off.y / p.p[3]);
        t = length(nrm);
    }
    if (p.stops.empty()) return;
    if (t < p.stops[0].offset) {
        add_stop_color(g, sb, 0, d_color);
        return;
    }
    for (size_t i = 0; i + 1 < p.stops.size(); ++i) {
        const Stop& cu = p.stops[i];
        const Stop& nx = p.stops[i + 1];
        if (t >= cu.offset && t < nx.offset) {
            float tt = (t - cu.offset) / (nx.offset - cu.offset);
            V4 cc = V4{cu.color.r, cu.color.g, cu.color.b, cu.color.a};
            V4 cn = V4{nx.color.r, nx.color.g, nx.color.b, nx.color.a};
            add_stop_color(g, sb, i, V4{d_color.x * (1.0f - tt), d_color.y * (1.0f - tt), d_color.z * (1.0f - tt),
                                        d_color.w * (1.0f - tt)});
            add_stop_color(g, sb, i + 1, V4{d_color.x * tt, d_color.y * tt, d_color.z * tt, d_color.w * tt});
            V4 diff = V4{cn.x - cc.x, cn.y - cc.y, cn.z - cc.z, cn.w - cc.w};
            float d_tt = dot4(d_color, diff);
            float denom_offset = nx.offset - cu.offset;
            if (std::fabs(denom_offset) > 0.0f) {
                float d_offset_next = -d_tt * tt / denom_offset;
                float d_offset_curr = d_tt * (tt - 1.0f) / denom_offset;
                g.stop_offsets[sb + i] += d_offset_curr;
                g.stop_offsets[sb + i + 1] += d_offset_next;
            }
            float d_t = d_tt / denom_offset;
            if (p.kind == DVG_PAINT_LINEAR) {
                V2 d_beg = mk(d_t * (-(pt.x - beg.x) - (end.x - beg.x)) / denom,
                              d_t * (-(pt.y - beg.y) - (end.y - beg.y)) / denom);
                V2 d_end = mk(d_t * (pt.x - beg.x) / denom, d_t * (pt.y - beg.y) / denom);
                float d_l = -d_t * t / denom;
                if (dot(end - beg, end - beg) > 1.0e-3f) {
                    V2 adjust = mk(beg.x - end.x, beg.y - end.y);
                    V2 ds = mk(d_beg.x + 2.0f * d_l * adjust.x, d_beg.y + 2.0f * d_l * adjust.y);
                    V2 de = mk(d_end.x + 2.0f * d_l * (end.x - beg.x), d_end.y + 2.0f * d_l * (end.y - beg.y));
                    dp[0] += ds.x;
                    dp[1] += ds.y;
                    dp[2] += de.x;
                    dp[3] += de.y;
                } else {
                    dp[0] += d_beg.x;
                    dp[1] += d_beg.y;
                    dp[2] += d_end.x;
                    dp[3] += d_end.y;
                }
                *d_translation += d_beg + d_end;
            } else {
                V2 d_nrm = d_length(nrm, d_t);
                V2 d_off = mk(d_nrm.x / p.p[2], d_nrm.y / p.p[3]);
                V2 d_radius = mk(-d_nrm.x * off.x / (p.p[2] * p.p[2]), -d_nrm.y * off.y / (p.p[3] * p.p[3]));
                V2 d_center = mk(-d_off.x, -d_off.y);
                dp[0] += d_center.x;
                dp[1] += d_center.y;
                dp[2] += d_radius.x;
                dp[3] += d_radius.y;
                *d_translation += d_center;
            }
            return;
        }
    }
    add_stop_color(g, sb, p.stops.size() - 1, d_color);
}

// ---------------------------------------------------------------- background (backward/background.rs)
static V4 sample_background(const Scene& sc, size_t pixel_index) {  // background.rs:7-26
    if (sc.has_bg_img) {
        size_t base = pixel_index * 4;
        if (base + 3 >= sc.bg_img.size()) return V4{0, 0, 0, 0};
        float r = sc.bg_img[base], g = sc.bg_img[base + 1], b = sc.bg_img[base + 2], a = sc.bg_img[base + 3];
        return V4{r * a, g * a, b * a, a};
    }
    return V4{sc.bg.r * sc.bg.a, sc.bg.g * sc.bg.a, sc.bg.b * sc.bg.a, sc.bg.a};
}
static void accumulate_background_grad(const Scene& sc, Grads& g, size_t pixel_index, V4 d) {  // background.rs:64-90
    if (sc.has_bg_img) {
        if (g.has_bg_image) {
            size_t base = pixel_index * 4;
            if (base + 3 < g.bg_image.size()) {
                g.bg_image[base] += d.x;
                g.bg_image[base + 1] += d.y;
                g.bg_image[base + 2] += d.z;
                g.bg_image[base + 3] += d.w;
            }
        }
        return;
    }
    g.background[0] = g.background[0] + d.x;
    g.background[1] = g.background[1] + d.y;
    g.background[2] = g.background[2] + d.z;
    g.background[3] = g.background[3] + d.w;
}
static void finalize_background_gradients(const Scene& sc, Grads& g) {  // background.rs:29-61
    if (sc.has_bg_img) {
        if (g.has_bg_image) {
            for (size_t i = 0; i * 4 < g.bg_image.size(); ++i) {
                size_t base = i * 4;
                float r = sc.bg_img[base], gg = sc.bg_img[base + 1], b = sc.bg_img[base + 2], a = sc.bg_img[base + 3];
                float* c = &g.bg_image[base];
                float dr = c[0] * a, dg = c[1] * a, db = c[2] * a;
                float da = c[0] * r + c[1] * gg + c[2] * b + c[3];
                c[0] = dr;
                c[1] = dg;
                c[2] = db;
                c[3] = da;
            }
        }
    } else {
        float r = sc.bg.r, gg = sc.bg.g, b = sc.bg.b, a = sc.bg.a;
        float* d = g.background;
        float nr = d[0] * a, ng = d[1] * a, nb = d[2] * a;
        float na = d[0] * r + d[1] * gg + d[2] * b + d[3];
        d[0] = nr;
        d[1] = ng;
        d[2] = nb;
        d[3] = na;
    }
}

// ---------------------------------------------------------------- filters (backward/filters.rs)
static float compute_filter_weight(uint32_t ft, float radius, float dx, float dy) {  // filters.rs:159-188
    if (radius <= 0.0f) return 1.0f;
    if (std::fabs(dx) > radius || std::fabs(dy) > radius) return 0.0f;
    switch (ft) {
        case DVG_FILTER_BOX:
            return 1.0f / ((2.0f * radius) * (2.0f * radius));
        case DVG_FILTER_TENT: {
            float fx = radius - std::fabs(dx), fy = radius - std::fabs(dy);
            float norm = 1.0f / (radius * radius);
            return fx * fy * norm * norm;
        }
        case DVG_FILTER_RADIAL_PARABOLIC: {
            float rx = 1.0f - (dx / radius) * (dx / radius);
            float ry = 1.0f - (dy / radius) * (dy / radius);
            return (4.0f / 3.0f) * rx * (4.0f / 3.0f) * ry;
        }
        case DVG_FILTER_HANN: {
            float ndx = (dx / (2.0f * radius)) + 0.5f, ndy = (dy / (2.0f * radius)) + 0.5f;
            float fx = 0.5f * (1.0f - std::cos(2.0f * PI_F * ndx));
            float fy = 0.5f * (1.0f - std::cos(2.0f * PI_F * ndy));
            float norm = 1.0f / (radius * radius);
            return fx * fy * norm;
        }
        case DVG_FILTER_GAUSSIAN: {
            // Addition of this library (not in the crate): normalised 2-D Gaussian with
            // sigma = radius/2 truncated to the square support |dx|,|dy| <= radius:
            // w = 2/(pi r^2) * exp(-2 (dx^2+dy^2) / r^2).
            float r2 = radius * radius;
            float q = dx * dx + dy * dy;
            return (2.0f / (PI_F * r2)) * std::exp(-2.0f * q / r2);
        }
        default:
            return 1.0f;
    }
}
static void d_compute_filter_weight(uint32_t ft, float radius, float dx, float dy, float d_return,
                                    float* d_radius) {  // filters.rs:190-239
    switch (ft) {
        case DVG_FILTER_BOX: {
            float denom = 2.0f * radius;
            if (denom != 0.0f) *d_radius += d_return * (-2.0f) * denom / ((denom * denom) * denom);
            break;
        }
        case DVG_FILTER_TENT: {
            float fx = radius - std::fabs(dx), fy = radius - std::fabs(dy);
            float norm = 1.0f / (radius * radius);
            float d_fx = d_return * fy * norm, d_fy = d_return * fx * norm, d_norm = d_return * fx * fy;
            float r2 = radius * radius;
            if (radius != 0.0f) *d_radius += d_fx + d_fy + (-4.0f) * d_norm / ((r2 * r2) * radius);
            break;
        }
        case DVG_FILTER_RADIAL_PARABOLIC: {
            float r3 = radius * radius * radius;
            if (r3 != 0.0f) *d_radius += -(2.0f * dx * dx + 2.0f * dy * dy) / r3;
            break;
        }
        case DVG_FILTER_HANN: {
            float ndx = (dx / (2.0f * radius)) + 0.5f, ndy = (dy / (2.0f * radius)) + 0.5f;
            float fx = 0.5f * (1.0f - std::cos(2.0f * PI_F * ndx));
            float fy = 0.5f * (1.0f - std::cos(2.0f * PI_F * ndy));
            float norm = 1.0f / (radius * radius);
            float d_fx = d_return * fy * norm, d_fy = d_return * fx * norm, d_norm = d_return * fx * fy;
            float d_ndx = d_fx * 0.5f * std::sin(2.0f * PI_F * ndx) * (2.0f * PI_F);
            float d_ndy = d_fy * 0.5f * std::sin(2.0f * PI_F * ndy) * (2.0f * PI_F);
            float tr = 2.0f * radius;
            *d_radius += d_ndx * (-2.0f * dx / (tr * tr)) + d_ndy * (-2.0f * dy / (tr * tr)) +
                         (-2.0f) * d_norm / ((radius * radius) * radius);
            break;
        }
        case DVG_FILTER_GAUSSIAN: {
            // d/dr of 2/(pi r^2) exp(-2q/r^2) = w * (4q/r^3 - 2/r)
            float r2 = radius * radius;
            float q = dx * dx + dy * dy;
            float w = (2.0f / (PI_F * r2)) * std::exp(-2.0f * q / r2);
            if (radius != 0.0f) *d_radius += d_return * w * (4.0f * q / (r2 * radius) - 2.0f / radius);
            break;
        }
        default:
            break;
    }
}

// PCG32 (src/renderer/rng.rs:16-43)
struct Pcg32 {
    uint64_t state, inc;
    Pcg32(uint64_t idx, uint64_t seed) {
        state = 0;
        inc = ((idx + 1) << 1) | 1;
        next_u32();
        state = state + (0x853c49e6748fea9bULL + seed);
        next_u32();
    }
    uint32_t next_u32() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + (inc | 1);
        uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
    }
    float next_f32() {
        uint32_t u = next_u32();
        uint32_t bits = (u >> 9) | 0x3f800000u;
        float f;
        std::memcpy(&f, &bits, 4);
        return f - 1.0f;
    }
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy as
// 1, 2, 3", SC 2011): counter = (idx_lo, idx_hi, 0, 0), key = (seed, 0).
static void philox4x32_10(uint32_t ctr[4], uint32_t key[2]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * ctr[0];
        uint64_t p1 = (uint64_t)M1 * ctr[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ ctr[1] ^ k0, n1 = lo1, n2 = hi0 ^ ctr[3] ^ k1, n3 = lo0;
        ctr[0] = n0;
        ctr[1] = n1;
        ctr[2] = n2;
        ctr[3] = n3;
        k0 += W0;
        k1 += W1;
    }
}
static inline float u32_to_unit(uint32_t u) { return (float)(u >> 9) * (1.0f / 8388608.0f); }
static void boundary_rng(uint32_t kind, uint64_t idx, uint32_t seed, float* u, float* t) {
    if (kind == DVG_RNG_PHILOX) {
        uint32_t ctr[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), 0u, 0u};
        uint32_t key[2] = {seed, 0u};
        philox4x32_10(ctr, key);
        *u = u32_to_unit(ctr[0]);
        *t = u32_to_unit(ctr[1]);
        return;
    }
    Pcg32 rng(idx, (uint64_t)seed);
    *u = rng.next_f32();
    *t = rng.next_f32();
}

struct SampleSpec {
    uint32_t sx_n, sy_n;
    bool jitter;
    bool prefilter;
    uint32_t seed;
};
static void sample_position(const Scene& sc, const SampleSpec& sp, uint64_t idx, V2* pt, size_t* pixel) {  // render.rs:95-111
    uint64_t sx = idx % sp.sx_n;
    uint64_t sy = (idx / sp.sx_n) % sp.sy_n;
    uint64_t x = (idx / ((uint64_t)sp.sx_n * sp.sy_n)) % sc.w;
    uint64_t y = idx / ((uint64_t)sp.sx_n * sp.sy_n * sc.w);
    float rx = 0.5f, ry = 0.5f;
    if (sp.jitter) {
        Pcg32 rng(idx, (uint64_t)sp.seed);
        rx = rng.next_f32();
        ry = rng.next_f32();
    }
    if (sp.prefilter) {
        rx = 0.5f;
        ry = 0.5f;
    }
    float px = (float)x + ((float)sx + rx) / (float)sp.sx_n;
    float py = (float)y + ((float)sy + ry) / (float)sp.sy_n;
    *pt = mk(px, py);
    *pixel = (size_t)(y * sc.w + x);
}

static std::vector<float> build_weight_image(const Scene& sc, const SampleSpec& sp) {  // filters.rs:11-67
    int width = (int)sc.w, height = (int)sc.h;
    std::vector<float> wimg((size_t)width * height, 0.0f);
    uint64_t total = (uint64_t)width * height * sp.sx_n * sp.sy_n;
    int ri = to_i32(std::ceil(sc.filter_radius));
    for (uint64_t idx = 0; idx < total; ++idx) {
        V2 pt;
        size_t pix;
        sample_position(sc, sp, idx, &pt, &pix);
        int x = (int)(pix % sc.w), y = (int)(pix / sc.w);
        for (int dy = -ri; dy <= ri; ++dy)
            for (int dx = -ri; dx <= ri; ++dx) {
                int xx = x + dx, yy = y + dy;
                if (xx >= 0 && yy >= 0 && xx < width && yy < height) {
                    float xc = (float)xx + 0.5f, yc = (float)yy + 0.5f;
                    float w = compute_filter_weight(sc.filter_type, sc.filter_radius, xc - pt.x, yc - pt.y);
                    wimg[(size_t)yy * width + xx] += w;
                }
            }
    }
    return wimg;
}
static V4 gather_d_color(const Scene& sc, const float* d_render, const std::vector<float>& wimg, V2 pt) {  // filters.rs:70-103
    int width = (int)sc.w, height = (int)sc.h;
    int x = to_i32(std::floor(pt.x)), y = to_i32(std::floor(pt.y));
    int ri = to_i32(std::ceil(sc.filter_radius));
    V4 out{0, 0, 0, 0};
    for (int dy = -ri; dy <= ri; ++dy)
        for (int dx = -ri; dx <= ri; ++dx) {
            int xx = x + dx, yy = y + dy;
            if (xx >= 0 && yy >= 0 && xx < width && yy < height) {
                float xc = (float)xx + 0.5f, yc = (float)yy + 0.5f;
                float w = compute_filter_weight(sc.filter_type, sc.filter_radius, xc - pt.x, yc - pt.y);
                float ws = wimg[(size_t)yy * width + xx];
                if (ws > 0.0f) {
                    size_t base = ((size_t)yy * width + xx) * 4;
                    out.x += (w / ws) * d_render[base];
                    out.y += (w / ws) * d_render[base + 1];
                    out.z += (w / ws) * d_render[base + 2];
                    out.w += (w / ws) * d_render[base + 3];
                }
            }
        }
    return out;
}
static void accumulate_filter_gradient(const Scene& sc, V4 color, const float* d_render,
                                       const std::vector<float>& wimg, V2 pt, float* d_radius) {  // filters.rs:106-156
    int width = (int)sc.w, height = (int)sc.h;
    int x = to_i32(std::floor(pt.x)), y = to_i32(std::floor(pt.y));
    int ri = to_i32(std::ceil(sc.filter_radius));
    for (int dy = -ri; dy <= ri; ++dy)
        for (int dx = -ri; dx <= ri; ++dx) {
            int xx = x + dx, yy = y + dy;
            if (xx >= 0 && yy >= 0 && xx < width && yy < height) {
                float ws = wimg[(size_t)yy * width + xx];
                if (ws <= 0.0f) continue;
                float xc = (float)xx + 0.5f, yc = (float)yy + 0.5f;
                float w = compute_filter_weight(sc.filter_type, sc.filter_radius, xc - pt.x, yc - pt.y);
                if (w <= 0.0f) continue;
                size_t base = ((size_t)yy * width + xx) * 4;
                V4 dpx{d_render[base], d_render[base + 1], d_render[base + 2], d_render[base + 3]};
                float dt = dot4(dpx, color);
                float denom = ws * ws;
                float d_weight = denom > 0.0f ? (dt * ws - w * dt * (ws - w)) / denom : 0.0f;
                if (d_weight != 0.0f)
                    d_compute_filter_weight(sc.filter_type, sc.filter_radius, xc - pt.x, yc - pt.y, d_weight,
                                            d_radius);
            }
        }
}

// ---------------------------------------------------------------- sample colour (backward/sampling.rs)
struct EdgeQuery {  // types.rs:42-50
    size_t group_id, shape_id;
    bool hit;
};
struct Fragment {  // types.rs:105-115
    float r, g, b, a;
    size_t group_id;
    bool is_stroke;
};
static bool within_distance_edge(const Scene& sc, const SceneBvh& bvh, size_t gi, V2 pt, EdgeQuery* eq) {  // sampling.rs:485-513
    bool hit = within_distance_bvh(sc, bvh, gi, pt);
    if (!eq || eq->group_id != gi) return hit;
    if (gi >= sc.groups.size() || eq->shape_id >= sc.shapes.size()) return hit;
    const Shape& s = sc.shapes[eq->shape_id];
    if (s.stroke_width <= 0.0f) return hit;
    V2 lp = xform_pt(sc.groups[gi].c2s, pt);
    if (within_distance_shape(s, lp, s.stroke_width)) eq->hit = true;
    return hit;
}
static bool is_inside_edge(const Scene& sc, const SceneBvh& bvh, size_t gi, V2 pt, EdgeQuery* eq) {  // sampling.rs:516-552
    bool inside = is_inside_bvh(sc, bvh, gi, pt);
    if (!eq || eq->group_id != gi) return inside;
    if (gi >= sc.groups.size() || eq->shape_id >= sc.shapes.size()) return inside;
    const Group& g = sc.groups[gi];
    const Shape& s = sc.shapes[eq->shape_id];
    V2 lp = xform_pt(g.c2s, pt);
    V2 sp = xform_inv_bwd(s.transform, lp);
    const PathBvh* pb = nullptr;
    if (gi < bvh.groups.size())
        for (const BvhShape& bs : bvh.groups[gi].shapes)
            if (bs.shape_index == eq->shape_id) {
                pb = bs.has_path_bvh ? &bs.path_bvh : nullptr;
                break;
            }
    int winding = winding_number_shape(s, pb, sp);
    if (fill_rule_hit(g.fill_rule, winding)) eq->hit = true;
    return inside;
}
static void accumulate_translation(Grads& g, long translation_index, V2 delta) {  // sampling.rs:555-563
    if (translation_index >= 0 && g.has_translation) {
        size_t idx = (size_t)translation_index * 2;
        g.translation[idx] += delta.x;
        g.translation[idx + 1] += delta.y;
    }
}

// Collect fragments (stroke then fill per group, in group order) — sampling.rs:91-119.
static void collect_fragments(const Scene& sc, const SceneBvh& bvh, V2 pt, EdgeQuery* eq,
                              std::vector<Fragment>& frags) {
    frags.clear();
    for (size_t gi = 0; gi < sc.groups.size(); ++gi) {
        const Group& g = sc.groups[gi];
        if (g.stroke >= 0) {
            if (within_distance_edge(sc, bvh, gi, pt, eq)) {
                V4 c = paint_color(sc.paints[g.stroke], pt);
                frags.push_back(Fragment{c.x, c.y, c.z, c.w, gi, true});
            }
        }
        if (g.fill >= 0) {
            if (is_inside_edge(sc, bvh, gi, pt, eq)) {
                V4 c = paint_color(sc.paints[g.fill], pt);
                frags.push_back(Fragment{c.x, c.y, c.z, c.w, gi, false});
            }
        }
    }
}

// sample_color (sampling.rs:76-224).  screen_pt is in normalised [0,1] canvas units.
static V4 sample_color(const Scene& sc, const SceneBvh& bvh, V2 screen_pt, const V4* background,
                       const V4* d_color, EdgeQuery* eq, Grads* grads, long translation_index,
                       size_t pixel_index) {
    if (eq) eq->hit = false;
    V2 pt = mk(screen_pt.x * (float)sc.w, screen_pt.y * (float)sc.h);
    std::vector<Fragment> frags;
    collect_fragments(sc, bvh, pt, eq, frags);
    if (frags.empty()) {
        if (background) {
            if (d_color) accumulate_background_grad(sc, *grads, pixel_index, *d_color);
            return *background;
        }
        return V4{0, 0, 0, 0};
    }
    // fragments are produced in ascending group order already (stable sort is a no-op)
    std::vector<V4> accum(frags.size());
    float pr = 0, pg = 0, pb = 0, pa = 0;
    if (background) {
        pr = background->x;
        pg = background->y;
        pb = background->z;
        pa = background->w;
    }
    for (size_t i = 0; i < frags.size(); ++i) {
        const Fragment& f = frags[i];
        if (eq) {
            if (f.a >= 1.0f && eq->hit) eq->hit = false;
            if (eq->group_id == f.group_id) eq->hit = true;
        }
        float br = pr * (1.0f - f.a) + f.r * f.a;
        float bg = pg * (1.0f - f.a) + f.g * f.a;
        float bb = pb * (1.0f - f.a) + f.b * f.a;
        float ba = pa * (1.0f - f.a) + f.a;
        accum[i] = V4{br, bg, bb, ba};
        pr = br;
        pg = bg;
        pb = bb;
        pa = ba;
    }
    V4 fc = accum.back();
    float final_alpha = fc.w;
    float fr = fc.x, fg = fc.y, fb = fc.z;
    if (final_alpha > 1.0e-6f) {
        float s = 1.0f / final_alpha;
        fr = fr * s;
        fg = fg * s;
        fb = fb * s;
    }
    if (d_color) {
        float dcr = d_color->x, dcg = d_color->y, dcb = d_color->z, dca = d_color->w;
        if (final_alpha > 1.0e-6f) {
            float dfr = dcr, dfg = dcg, dfb = dcb;
            float s = 1.0f / final_alpha;
            dcr = dcr * s;
            dcg = dcg * s;
            dcb = dcb * s;
            dca -= (dfr * fr + dfg * fg + dfb * fb) / final_alpha;
        }
        for (size_t ii = frags.size(); ii-- > 0;) {
            float prev_a, prev_r, prev_g, prev_b;
            if (ii > 0) {
                prev_a = accum[ii - 1].w;
                prev_r = accum[ii - 1].x;
                prev_g = accum[ii - 1].y;
                prev_b = accum[ii - 1].z;
            } else {
                prev_a = background ? background->w : 0.0f;
                prev_r = background ? background->x : 0.0f;
                prev_g = background ? background->y : 0.0f;
                prev_b = background ? background->z : 0.0f;
            }
            const Fragment& f = frags[ii];
            float d_prev_alpha = dca * (1.0f - f.a);
            float d_alpha_i = dca * (1.0f - prev_a);
            d_alpha_i += dcr * (f.r - prev_r) + dcg * (f.g - prev_g) + dcb * (f.b - prev_b);
            float s = 1.0f - f.a;
            float dpr = dcr * s, dpg = dcg * s, dpb = dcb * s;
            V4 dv{dcr * f.a, dcg * f.a, dcb * f.a, d_alpha_i};
            V2 tdelta = mk(0, 0);
            const Group& g = sc.groups[f.group_id];
            int pi = f.is_stroke ? g.stroke : g.fill;
            if (pi >= 0) d_sample_paint(sc, pi, *grads, pt, dv, &tdelta);
            accumulate_translation(*grads, translation_index, tdelta);
            dcr = dpr;
            dcg = dpg;
            dcb = dpb;
            dca = d_prev_alpha;
        }
        if (background) accumulate_background_grad(sc, *grads, pixel_index, V4{dcr, dcg, dcb, dca});
    }
    return V4{fr, fg, fb, final_alpha};
}

// ---------------------------------------------------------------- prefiltered sampling (backward/sampling.rs:227-482)
struct PathInfo {  // types.rs:33-41
    bool valid = false;
    size_t base_point_id = 0, point_id = 0;
    float t = 0.0f;
};
static size_t path_point_id(const PathG& p, size_t base_point_id) {  // backward/distance.rs:35-47
    size_t point_id = 0;
    size_t count = std::min(base_point_id, p.ncp.size());
    for (size_t i = 0; i < count; ++i) {
        uint8_t c = p.ncp[i];
        point_id += c == 0 ? 1 : (c == 1 ? 2 : (c == 2 ? 3 : 0));
    }
    return point_id;
}
static PathInfo path_info_from_closest(const Scene& sc, size_t shape_index, const PathHit& h) {  // distance.rs:14-32
    PathInfo pi;
    if (sc.shapes[shape_index].kind != DVG_SHAPE_PATH || !h.valid) return pi;
    pi.valid = true;
    pi.base_point_id = h.segment_index;
    pi.point_id = path_point_id(sc.shapes[shape_index].path, h.segment_index);
    pi.t = h.t;
    return pi;
}
static float d_smoothstep(float d, float d_ret) {  // backward/math.rs:15-22
    if (d < -1.0f || d > 1.0f) return 0.0f;
    float t = (d + 1.0f) * 0.5f;
    float d_t = d_ret * (6.0f * t - 6.0f * t * t);
    return d_t * 0.5f;
}
static void d_distance(V2 a, V2 b, float d_out, V2* d_a, V2* d_b) {  // math.rs:25-30
    V2 d = d_length(b - a, d_out);
    *d_a -= d;
    *d_b += d;
}
static V2 d_normalize(V2 v, V2 d_n) {  // math.rs:53-63
    float l = length(v);
    if (l == 0.0f) return mk(0, 0);
    V2 n = v / l;
    V2 d_v = d_n / l;
    float d_l = -dot(d_n, n) / l;
    d_v += d_length(v, d_l);
    return d_v;
}
static M3 scale3(const M3& m, float s) {
    M3 o = m;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o.m[r][c] *= s;
    return o;
}
static M3 add3(const M3& a, const M3& b) {
    M3 o = a;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o.m[r][c] += b.m[r][c];
    return o;
}
static void add_shape_transform(Grads& g, size_t shape_id, const M3& m) {
    float* ds = &g.shape_transform[9 * shape_id];
    for (int i = 0; i < 9; ++i) ds[i] = ds[i] + m.m[i / 3][i % 3];
}
static void add_group_transform(Grads& g, size_t group_id, const M3& m) {
    float* dg = &g.group_transform[9 * group_id];
    for (int i = 0; i < 9; ++i) dg[i] = dg[i] + m.m[i / 3][i % 3];
}
static void d_closest_point_path(const Shape& s, size_t shape_id, V2 pt, V2 d_cp, const PathInfo& info, Grads& g,
                                 V2* d_pt) {  // backward/distance.rs:190-394
    const PathG& path = s.path;
    size_t bpid = info.base_point_id, pid = info.point_id;
    float min_t = info.t;
    size_t np = path.pts.size();
    if (np == 0) return;
    auto get_point = [&](size_t idx) { return path.closed ? path.pts[idx % np] : path.pts[std::min(idx, np - 1)]; };
    auto add_point = [&](size_t idx, V2 delta) {
        size_t index = path.closed ? idx % np : idx;
        if (index < np) {
            g.points[2 * (path.point_base + index)] += delta.x;
            g.points[2 * (path.point_base + index) + 1] += delta.y;
        }
    };
    uint8_t nc = bpid < path.ncp.size() ? path.ncp[bpid] : 0;
    if (nc == 0) {
        size_t i0 = pid, i1 = (pid + 1) % np;
        V2 p0 = get_point(i0), p1 = get_point(i1);
        float t = dot(pt - p0, p1 - p0) / dot(p1 - p0, p1 - p0);
        if (t < 0.0f) {
            add_point(i0, d_cp);
        } else if (t > 1.0f) {
            add_point(i1, d_cp);
        } else {
            add_point(i0, d_cp * (1.0f - t));
            add_point(i1, d_cp * t);
        }
    } else if (nc == 1) {
        size_t i0 = pid, i1 = pid + 1, i2 = (pid + 2) % np;
        V2 p0 = get_point(i0), p1 = get_point(i1), p2 = get_point(i2);
        float t = min_t;
        V2 d_p0 = mk(0, 0), d_p1 = mk(0, 0), d_p2 = mk(0, 0);
        if (t == 0.0f) {
            d_p0 += d_cp;
        } else if (t == 1.0f) {
            d_p2 += d_cp;
        } else {
            V2 a = p0 - p1 * 2.0f + p2;
            V2 b = p1 - p0;
            float A = dot(a, a);
            float B = 3.0f * dot(a, b);
            float C = 2.0f * dot(b, b) + dot(a, p0 - pt);
            float tt = 1.0f - t;
            V2 d_p = d_cp;
            float d_tt = 2.0f * tt * dot(d_p, p0) + 2.0f * t * dot(d_p, p1);
            float d_t = -d_tt + 2.0f * tt * dot(d_p, p1) + 2.0f * t * dot(d_p, p2);
            d_p0 += d_p * (tt * tt);
            d_p1 += d_p * (2.0f * tt * t);
            d_p2 += d_p * (t * t);
            float poly_deriv_t = 3.0f * A * t * t + 2.0f * B * t + C;
            if (std::fabs(poly_deriv_t) > 1.0e-6f) {
                float d_A = -(d_t / poly_deriv_t) * t * t * t;
                float d_B = -(d_t / poly_deriv_t) * t * t;
                float d_C = -(d_t / poly_deriv_t) * t;
                float d_D = -(d_t / poly_deriv_t);
                d_p0 += a * (2.0f * d_A) + (b - a) * (3.0f * d_B) + (b * -4.0f) * d_C + (p0 - pt + a) * d_C +
                        (b - (p0 - pt)) * (2.0f * d_D);
                d_p1 += a * (-4.0f * d_A) + (a + b * -2.0f) * (3.0f * d_B) + (b * 4.0f) * d_C +
                        (p0 - pt) * (-2.0f * d_C) + (p0 - pt) * d_D;
                d_p2 += a * (2.0f * d_A) + b * (3.0f * d_B) + (p0 - pt) * d_C;
                *d_pt += a * (-d_C) + b * d_D;
            }
        }
        add_point(i0, d_p0);
        add_point(i1, d_p1);
        add_point(i2, d_p2);
    } else if (nc == 2) {
        size_t i0 = pid, i1 = pid + 1, i2 = pid + 2, i3 = (pid + 3) % np;
        V2 p0 = get_point(i0), p1 = get_point(i1), p2 = get_point(i2), p3 = get_point(i3);
        float t = min_t;
        V2 d_p0 = mk(0, 0), d_p1 = mk(0, 0), d_p2 = mk(0, 0), d_p3 = mk(0, 0);
        if (t == 0.0f) {
            d_p0 += d_cp;
        } else if (t == 1.0f) {
            d_p3 += d_cp;
        } else {
            V2 a = p0 * -1.0f + p1 * 3.0f + p2 * -3.0f + p3;
            V2 b = p0 * 3.0f + p1 * -6.0f + p2 * 3.0f;
            V2 c = p0 * -3.0f + p1 * 3.0f;
            float A = 3.0f * dot(a, a);
            if (std::fabs(A) < 1.0e-10f) return;
            float B = 5.0f * dot(a, b);
            float C = 4.0f * dot(a, c) + 2.0f * dot(b, b);
            float D = 3.0f * (dot(b, c) + dot(a, p0 - pt));
            float E = dot(c, c) + 2.0f * dot(p0 - pt, b);
            float F = dot(p0 - pt, c);
            B = B / A;
            C = C / A;
            D = D / A;
            E = E / A;
            F = F / A;
            float tt = 1.0f - t;
            V2 d_p = d_cp;
            float d_tt = 3.0f * tt * tt * dot(d_p, p0) + 6.0f * tt * t * dot(d_p, p1) + 3.0f * t * t * dot(d_p, p2);
            float d_t = -d_tt + 3.0f * tt * tt * dot(d_p, p1) + 6.0f * tt * t * dot(d_p, p2) +
                        3.0f * t * t * dot(d_p, p3);
            d_p0 += d_p * (tt * tt * tt);
            d_p1 += d_p * (3.0f * tt * tt * t);
            d_p2 += d_p * (3.0f * tt * t * t);
            d_p3 += d_p * (t * t * t);
            float pd = 5.0f * t * t * t * t + 4.0f * B * t * t * t + 3.0f * C * t * t + 2.0f * D * t + E;
            if (std::fabs(pd) > 1.0e-10f) {
                float d_B = -(d_t / pd) * t * t * t * t;
                float d_C = -(d_t / pd) * t * t * t;
                float d_D = -(d_t / pd) * t * t;
                float d_E = -(d_t / pd) * t;
                float d_F = -(d_t / pd);
                float d_A = -d_B * B / A - d_C * C / A - d_D * D / A - d_E * E / A - d_F * F / A;
                d_B /= A;
                d_C /= A;
                d_D /= A;
                d_E /= A;
                d_F /= A;
                d_p0 += a * (3.0f * -1.0f * 2.0f * d_A);
                d_p1 += a * (3.0f * 3.0f * 2.0f * d_A);
                d_p2 += a * (3.0f * -3.0f * 2.0f * d_A);
                d_p3 += a * (3.0f * 1.0f * 2.0f * d_A);
                d_p0 += (b * -1.0f + a * 3.0f) * (5.0f * d_B);
                d_p1 += (b * 3.0f + a * -6.0f) * (5.0f * d_B);
                d_p2 += (b * -3.0f + a * 3.0f) * (5.0f * d_B);
                d_p3 += b * (5.0f * d_B);
                d_p0 += (c * -1.0f + a * -3.0f) * (4.0f * d_C) + b * (3.0f * 2.0f * d_C);
                d_p1 += (c * 3.0f + a * 3.0f) * (4.0f * d_C) + b * (-6.0f * 2.0f * d_C);
                d_p2 += c * (-3.0f * d_C * 4.0f) + b * (3.0f * 2.0f * d_C);
                d_p3 += c * (4.0f * d_C);
                d_p0 += (c * 3.0f + b * -3.0f) * (3.0f * d_D) + (a - (p0 - pt)) * (3.0f * d_D);
                d_p1 += (c * -6.0f + b * 3.0f) * (3.0f * d_D) + (p0 - pt) * (3.0f * 3.0f * d_D);
                d_p2 += c * (3.0f * 3.0f * d_D) + (p0 - pt) * (-3.0f * 3.0f * d_D);
                *d_pt += a * (-1.0f * 3.0f * d_D);
                d_p0 += c * (-3.0f * 2.0f * d_E) + (b + (p0 - pt) * 3.0f) * (2.0f * d_E);
                d_p1 += c * (3.0f * 2.0f * d_E) + (p0 - pt) * (-6.0f * 2.0f * d_E);
                d_p2 += (p0 - pt) * (3.0f * 2.0f * d_E);
                *d_pt += b * (-1.0f * 2.0f * d_E);
                d_p0 += c * d_F + (p0 - pt) * (-3.0f * d_F);
                d_p1 += (p0 - pt) * (3.0f * d_F);
                *d_pt += c * (-1.0f * d_F);
            }
        }
        add_point(i0, d_p0);
        add_point(i1, d_p1);
        add_point(i2, d_p2);
        add_point(i3, d_p3);
    }
    (void)shape_id;
}
static void d_closest_point_rect(V2 mn, V2 mx, V2 pt, V2 d_cp, V2* d_min, V2* d_max, V2* d_pt) {  // distance.rs:397-476
    auto dist_to_seg = [&](V2 p0, V2 p1) {
        float t = dot(pt - p0, p1 - p0) / dot(p1 - p0, p1 - p0);
        if (t < 0.0f) return length(p0 - pt);
        if (t > 1.0f) return length(p1 - pt);
        return length(p0 + (p1 - p0) * t - pt);
    };
    V2 lt = mn, rt = mk(mx.x, mn.y), lb = mk(mn.x, mx.y), rb = mx;
    int min_id = 0;
    float min_dist = dist_to_seg(lt, lb);
    float top = dist_to_seg(lt, rt), right = dist_to_seg(rt, rb), bottom = dist_to_seg(lb, rb);
    if (top < min_dist) {
        min_dist = top;
        min_id = 1;
    }
    if (right < min_dist) {
        min_dist = right;
        min_id = 2;
    }
    if (bottom < min_dist) {
        min_dist = bottom;
        min_id = 3;
    }
    auto update = [&](V2 p0, V2 p1, V2* d_p0, V2* d_p1) {
        float t = dot(pt - p0, p1 - p0) / dot(p1 - p0, p1 - p0);
        if (t < 0.0f) {
            *d_p0 += d_cp;
        } else if (t > 1.0f) {
            *d_p1 += d_cp;
        } else {
            V2 d_p = d_cp;
            *d_p0 += d_p * (1.0f - t);
            *d_p1 += d_p * t;
            float d_t = dot(d_p, p1 - p0);
            float denom = dot(p1 - p0, p1 - p0);
            float d_num = d_t / denom;
            float d_den = d_t * (-t) / denom;
            *d_pt += (p1 - p0) * d_num;
            *d_p1 += (pt - p0) * d_num;
            *d_p0 += (p0 - p1 + p0 - pt) * d_num;
            *d_p1 += (p1 - p0) * (2.0f * d_den);
            *d_p0 += (p0 - p1) * (2.0f * d_den);
        }
    };
    V2 d_lt = mk(0, 0), d_rt = mk(0, 0), d_lb = mk(0, 0), d_rb = mk(0, 0);
    if (min_id == 0)
        update(lt, lb, &d_lt, &d_lb);
    else if (min_id == 1)
        update(lt, rt, &d_lt, &d_rt);
    else if (min_id == 2)
        update(rt, rb, &d_rt, &d_rb);
    else
        update(lb, rb, &d_lb, &d_rb);
    *d_min += d_lt;
    d_max->x += d_rt.x;
    d_min->y += d_rt.y;
    d_min->x += d_lb.x;
    d_max->y += d_lb.y;
    *d_max += d_rb;
}
static void d_closest_point_ellipse(V2 center, V2 radius, V2 pt, V2 d_cp, V2* d_center, V2* d_radius,
                                    V2* d_pt) {  // distance.rs:479-561
    float rx = std::fabs(radius.x), ry = std::fabs(radius.y);
    const float eps = 1.0e-6f;
    V2 local = pt - center;
    if (rx < eps && ry < eps) {
        *d_center += d_cp;
        return;
    }
    if (rx < eps) {
        float hit = (local.y >= -ry && local.y <= ry) ? 1.0f : 0.0f;
        *d_center += mk(d_cp.x, d_cp.y);
        d_pt->y += d_cp.y * hit;
        if (local.y > ry)
            d_radius->y += d_cp.y;
        else if (local.y < -ry)
            d_radius->y -= d_cp.y;
        return;
    }
    if (ry < eps) {
        float hit = (local.x >= -rx && local.x <= rx) ? 1.0f : 0.0f;
        *d_center += mk(d_cp.x, d_cp.y);
        d_pt->x += d_cp.x * hit;
        if (local.x > rx)
            d_radius->x += d_cp.x;
        else if (local.x < -rx)
            d_radius->x -= d_cp.x;
        return;
    }
    float sign_x = local.x < 0.0f ? -1.0f : 1.0f, sign_y = local.y < 0.0f ? -1.0f : 1.0f;
    float x = std::fabs(local.x), y = std::fabs(local.y);
    float t = std::atan2(y * rx, x * ry);
    float g_t = 0.0f;
    for (int i = 0; i < 20; ++i) {
        float sn = std::sin(t), cs = std::cos(t);
        float gg = rx * x * sn - ry * y * cs + (ry * ry - rx * rx) * sn * cs;
        g_t = rx * x * cs + ry * y * sn + (ry * ry - rx * rx) * (cs * cs - sn * sn);
        if (std::fabs(g_t) < 1.0e-12f) break;
        float next = clampf(t - gg / g_t, 0.0f, FRAC_PI_2_F);
        if (std::fabs(next - t) < 1.0e-6f) {
            t = next;
            break;
        }
        t = next;
    }
    float sn = std::sin(t), cs = std::cos(t);
    float d_t = 0.0f;
    d_radius->x += d_cp.x * sign_x * cs;
    d_t += d_cp.x * sign_x * (-rx * sn);
    d_radius->y += d_cp.y * sign_y * sn;
    d_t += d_cp.y * sign_y * (ry * cs);
    float g_a = x * sn - 2.0f * rx * sn * cs;
    float g_b = -y * cs + 2.0f * ry * sn * cs;
    float g_x = rx * sn;
    float g_y = -ry * cs;
    if (std::fabs(g_t) > 1.0e-12f) {
        float inv = -d_t / g_t;
        d_radius->x += inv * g_a;
        d_radius->y += inv * g_b;
        float d_x = inv * g_x, d_y = inv * g_y;
        d_pt->x += d_x * sign_x;
        d_pt->y += d_y * sign_y;
        d_center->x -= d_x * sign_x;
        d_center->y -= d_y * sign_y;
    }
}
static void d_closest_point(const Shape& s, size_t shape_id, V2 pt, V2 d_cp, const PathInfo& pinfo, Grads& g,
                            V2* d_pt) {  // distance.rs:139-187
    float* dp = &g.shape_params[4 * shape_id];
    if (s.kind == DVG_SHAPE_CIRCLE) {
        V2 center = mk(s.prm[0], s.prm[1]);
        float radius = s.prm[2];
        V2 v = pt - center;
        V2 n = normalize(v);
        V2 d_center = d_cp;
        float d_radius = dot(d_cp, n);
        V2 d_n = d_cp * radius;
        V2 d_v = d_normalize(v, d_n);
        d_center -= d_v;
        *d_pt += d_v;
        dp[0] += d_center.x;
        dp[1] += d_center.y;
        dp[2] += d_radius;
    } else if (s.kind == DVG_SHAPE_ELLIPSE) {
        V2 dc = mk(0, 0), dr = mk(0, 0);
        d_closest_point_ellipse(mk(s.prm[0], s.prm[1]), mk(s.prm[2], s.prm[3]), pt, d_cp, &dc, &dr, d_pt);
        dp[0] += dc.x;
        dp[1] += dc.y;
        dp[2] += dr.x;
        dp[3] += dr.y;
    } else if (s.kind == DVG_SHAPE_RECT) {
        V2 dmn = mk(0, 0), dmx = mk(0, 0);
        d_closest_point_rect(mk(s.prm[0], s.prm[1]), mk(s.prm[2], s.prm[3]), pt, d_cp, &dmn, &dmx, d_pt);
        dp[0] += dmn.x;
        dp[1] += dmn.y;
        dp[2] += dmx.x;
        dp[3] += dmx.y;
    } else if (s.kind == DVG_SHAPE_PATH) {
        if (!pinfo.valid) return;
        d_closest_point_path(s, shape_id, pt, d_cp, pinfo, g, d_pt);
    }
}
static V2 d_compute_distance(const Group& grp, size_t group_id, const Shape& s, size_t shape_id, V2 pt, V2 closest_pt,
                             const PathInfo& pinfo, float d_dist, Grads& g) {  // distance.rs:50-136
    if (length_sq(pt - closest_pt) < 1.0e-10f) return mk(0, 0);
    V2 lpg = xform_pt(grp.c2s, pt);
    V2 lcg = xform_pt(grp.c2s, closest_pt);
    M3 shape_inv;
    if (!inverse3(s.transform, &shape_inv)) shape_inv = identity3();
    V2 lps = xform_pt(shape_inv, lpg);
    V2 lcs = xform_pt(shape_inv, lcg);
    V2 d_pt = mk(0, 0), d_closest = mk(0, 0);
    d_distance(closest_pt, pt, d_dist, &d_closest, &d_pt);
    M3 d_s2c = zero3();
    V2 d_lcg = mk(0, 0);
    d_xform_pt(grp.s2c, lcg, d_closest, &d_s2c, &d_lcg);
    M3 d_st = zero3();
    V2 d_lcs = mk(0, 0);
    d_xform_pt(s.transform, lcs, d_lcg, &d_st, &d_lcs);
    V2 d_lps = mk(0, 0);
    d_closest_point(s, shape_id, lps, d_lcs, pinfo, g, &d_lps);
    M3 d_sinv = zero3();
    V2 d_lpg = mk(0, 0);
    d_xform_pt(shape_inv, lpg, d_lps, &d_sinv, &d_lpg);
    M3 d_c2s = zero3();
    d_xform_pt(grp.c2s, pt, d_lpg, &d_c2s, &d_pt);
    M3 tc2s = transpose3(grp.c2s);
    M3 corr = mul3(mul3(scale3(tc2s, -1.0f), d_c2s), tc2s);
    M3 dg = zero3();
    dg = add3(dg, d_s2c);
    dg = add3(dg, corr);
    add_group_transform(g, group_id, dg);
    M3 tsi = transpose3(shape_inv);
    M3 corr_s = mul3(mul3(scale3(tsi, -1.0f), d_sinv), tsi);
    M3 ds = zero3();
    ds = add3(ds, corr_s);
    ds = add3(ds, d_st);
    add_shape_transform(g, shape_id, ds);
    return d_pt;
}
struct PFrag {  // types.rs:118-136
    float r, g, b, a;
    size_t group_id, shape_id;
    float distance;
    V2 closest;
    PathInfo pinfo;
    bool within, is_stroke;
};
static bool styled_end_value(const Group& grp, const Shape& s, size_t seg, float t, V2 pt, float* sd);
static bool styled_end_backward(const Group& grp, size_t group_id, const Shape& s, size_t shape_id, size_t seg, float t,
                                V2 pt, float d_s, Grads& g, float* d_sw, V2* d_pt);
static void collect_prefiltered(const Scene& sc, const SceneBvh& bvh, V2 pt, std::vector<PFrag>& frags) {
    frags.clear();
    for (size_t gi = 0; gi < sc.groups.size(); ++gi) {
        const Group& g = sc.groups[gi];
        if (g.stroke >= 0) {
            ClosestPoint hit;
            if (compute_distance_bvh(sc, bvh, gi, pt, INF_F, &hit)) {
                const Shape& shp = sc.shapes[hit.shape_index];
                float d = hit.distance;
                float sd = 0.0f, w;
                if (hit.path.valid && (hit.path.t == 0.0f || hit.path.t == 1.0f) &&
                    styled_end_value(g, shp, hit.path.segment_index, hit.path.t, pt, &sd))
                    w = smoothstep(sd + 2.0f * shp.stroke_width) - smoothstep(sd);
                else
                    w = smoothstep(std::fabs(d) + shp.stroke_width) - smoothstep(std::fabs(d) - shp.stroke_width);
                if (w > 0.0f) {
                    V4 c = paint_color(sc.paints[g.stroke], pt);
                    c.w *= w;
                    frags.push_back(PFrag{c.x, c.y, c.z, c.w, gi, hit.shape_index, d, hit.point,
                                          path_info_from_closest(sc, hit.shape_index, hit.path), true, true});
                }
            }
        }
        if (g.fill >= 0) {
            ClosestPoint hit;
            bool have = compute_distance_bvh(sc, bvh, gi, pt, 1.0f, &hit);
            bool inside = is_inside_bvh(sc, bvh, gi, pt);
            if (have || inside) {
                size_t shape_id = 0;
                V2 cp = mk(0, 0);
                PathInfo pinfo;
                float d = 1.0f;
                if (have) {
                    shape_id = hit.shape_index;
                    cp = hit.point;
                    pinfo = path_info_from_closest(sc, hit.shape_index, hit.path);
                    d = hit.distance;
                }
                if (!inside) d = -d;
                float w = smoothstep(d);
                if (w > 0.0f) {
                    V4 c = paint_color(sc.paints[g.fill], pt);
                    c.w *= w;
                    frags.push_back(PFrag{c.x, c.y, c.z, c.w, gi, shape_id, d, cp, pinfo, have, false});
                }
            }
        }
    }
}
static V4 sample_color_prefiltered(const Scene& sc, const SceneBvh& bvh, V2 screen_pt, const V4* background,
                                   const V4* d_color, Grads* grads, long translation_index, size_t pixel_index) {
    V2 pt = mk(screen_pt.x * (float)sc.w, screen_pt.y * (float)sc.h);
    std::vector<PFrag> frags;
    collect_prefiltered(sc, bvh, pt, frags);
    if (frags.empty()) {
        if (background) {
            if (d_color) accumulate_background_grad(sc, *grads, pixel_index, *d_color);
            return *background;
        }
        return V4{0, 0, 0, 0};
    }
    std::vector<V4> accum(frags.size());
    float pr = 0, pg = 0, pb = 0, pa = 0;
    if (background) {
        pr = background->x;
        pg = background->y;
        pb = background->z;
        pa = background->w;
    }
    for (size_t i = 0; i < frags.size(); ++i) {
        const PFrag& f = frags[i];
        float br = pr * (1.0f - f.a) + f.r * f.a;
        float bg = pg * (1.0f - f.a) + f.g * f.a;
        float bb = pb * (1.0f - f.a) + f.b * f.a;
        float ba = pa * (1.0f - f.a) + f.a;
        accum[i] = V4{br, bg, bb, ba};
        pr = br;
        pg = bg;
        pb = bb;
        pa = ba;
    }
    V4 fc = accum.back();
    float final_alpha = fc.w, fr = fc.x, fg = fc.y, fb = fc.z;
    if (final_alpha > 1.0e-6f) {
        float s = 1.0f / final_alpha;
        fr = fr * s;
        fg = fg * s;
        fb = fb * s;
    }
    if (d_color) {
        float dcr = d_color->x, dcg = d_color->y, dcb = d_color->z, dca = d_color->w;
        if (final_alpha > 1.0e-6f) {
            float dfr = dcr, dfg = dcg, dfb = dcb;
            float s = 1.0f / final_alpha;
            dcr = dcr * s;
            dcg = dcg * s;
            dcb = dcb * s;
            dca -= (dfr * fr + dfg * fg + dfb * fb) / final_alpha;
        }
        for (size_t ii = frags.size(); ii-- > 0;) {
            float prev_a, prev_r, prev_g, prev_b;
            if (ii > 0) {
                prev_a = accum[ii - 1].w;
                prev_r = accum[ii - 1].x;
                prev_g = accum[ii - 1].y;
                prev_b = accum[ii - 1].z;
            } else {
                prev_a = background ? background->w : 0.0f;
                prev_r = background ? background->x : 0.0f;
                prev_g = background ? background->y : 0.0f;
                prev_b = background ? background->z : 0.0f;
            }
            const PFrag& f = frags[ii];
            float d_prev_alpha = dca * (1.0f - f.a);
            float d_alpha_i = dca * (1.0f - prev_a);
            d_alpha_i += dcr * (f.r - prev_r) + dcg * (f.g - prev_g) + dcb * (f.b - prev_b);
            float s = 1.0f - f.a;
            float dpr = dcr * s, dpg = dcg * s, dpb = dcb * s;
            float dci_r = dcr * f.a, dci_g = dcg * f.a, dci_b = dcb * f.a;
            const Group& grp = sc.groups[f.group_id];
            if (f.is_stroke) {
                const Shape& shp = sc.shapes[f.shape_id];
                float d = f.distance;
                float abs_plus = std::fabs(d) + shp.stroke_width, abs_minus = std::fabs(d) - shp.stroke_width;
                float sd = 0.0f;
                const bool styled = f.pinfo.valid && (f.pinfo.t == 0.0f || f.pinfo.t == 1.0f) &&
                                    styled_end_value(grp, shp, f.pinfo.base_point_id, f.pinfo.t, pt, &sd);
                float w = styled ? smoothstep(sd + 2.0f * shp.stroke_width) - smoothstep(sd)
                                 : smoothstep(abs_plus) - smoothstep(abs_minus);
                if (w != 0.0f && styled) {
                    float d_w = w > 0.0f ? (f.a / w) * d_alpha_i : 0.0f;
                    float dai = d_alpha_i * w;
                    V2 tdelta = mk(0, 0);
                    if (grp.stroke >= 0) d_sample_paint(sc, grp.stroke, *grads, pt, V4{dci_r, dci_g, dci_b, dai}, &tdelta);
                    float dp = d_smoothstep(sd + 2.0f * shp.stroke_width, d_w), dm = d_smoothstep(sd, d_w);
                    float d_s = dp - dm, d_sw = 0.0f;
                    V2 d_pt = mk(0, 0);
                    styled_end_backward(grp, f.group_id, shp, f.shape_id, f.pinfo.base_point_id, f.pinfo.t, pt, d_s,
                                        *grads, &d_sw, &d_pt);
                    grads->stroke_width[f.shape_id] += 2.0f * dp + d_sw;
                    accumulate_translation(*grads, translation_index, tdelta + d_pt * -1.0f);
                } else if (w != 0.0f) {
                    float d_w = w > 0.0f ? (f.a / w) * d_alpha_i : 0.0f;
                    float dai = d_alpha_i * w;
                    V2 tdelta = mk(0, 0);
                    if (grp.stroke >= 0) d_sample_paint(sc, grp.stroke, *grads, pt, V4{dci_r, dci_g, dci_b, dai}, &tdelta);
                    accumulate_translation(*grads, translation_index, tdelta);
                    float d_abs_plus = d_smoothstep(abs_plus, d_w);
                    float d_abs_minus = -d_smoothstep(abs_minus, d_w);
                    float d_d = d_abs_plus + d_abs_minus;
                    if (d < 0.0f) d_d = -d_d;
                    float d_sw = d_abs_plus - d_abs_minus;
                    grads->stroke_width[f.shape_id] += d_sw;
                    if (std::fabs(d_d) > 1.0e-10f) {
                        V2 d_pt = d_compute_distance(grp, f.group_id, shp, f.shape_id, pt, f.closest, f.pinfo, d_d,
                                                     *grads);
                        accumulate_translation(*grads, translation_index, d_pt * -1.0f);
                    }
                }
            } else {
                float d = f.distance;
                float w = smoothstep(d);
                if (w != 0.0f) {
                    float d_w = w > 0.0f ? (f.a / w) * d_alpha_i : 0.0f;
                    float dai = d_alpha_i * w;
                    V2 tdelta = mk(0, 0);
                    if (grp.fill >= 0) d_sample_paint(sc, grp.fill, *grads, pt, V4{dci_r, dci_g, dci_b, dai}, &tdelta);
                    accumulate_translation(*grads, translation_index, tdelta);
                    float d_d = d_smoothstep(d, d_w);
                    if (d < 0.0f) d_d = -d_d;
                    if (std::fabs(d_d) > 1.0e-10f && f.within) {
                        V2 d_pt = d_compute_distance(grp, f.group_id, sc.shapes[f.shape_id], f.shape_id, pt, f.closest,
                                                     f.pinfo, d_d, *grads);
                        accumulate_translation(*grads, translation_index, d_pt * -1.0f);
                    }
                }
            }
            dcr = dpr;
            dcg = dpg;
            dcb = dpb;
            dca = d_prev_alpha;
        }
        if (background) accumulate_background_grad(sc, *grads, pixel_index, V4{dcr, dcg, dcb, dca});
    }
    return V4{fr, fg, fb, final_alpha};
}
static V4 eval_premultiplied_prefiltered(const Scene& sc, const SceneBvh& bvh, V2 pt, V4 background) {
    std::vector<PFrag> frags;
    collect_prefiltered(sc, bvh, pt, frags);
    float pr = background.x, pg = background.y, pb = background.z, pa = background.w;
    for (const PFrag& f : frags) {
        float br = pr * (1.0f - f.a) + f.r * f.a;
        float bg = pg * (1.0f - f.a) + f.g * f.a;
        float bb = pb * (1.0f - f.a) + f.b * f.a;
        float ba = pa * (1.0f - f.a) + f.a;
        pr = br;
        pg = bg;
        pb = bb;
        pa = ba;
    }
    return V4{pr, pg, pb, pa};
}

// Premultiplied colour at canvas point pt (the crate's eval_scene_tiled output,
// src/gpu/kernels/forward.rs:1131-1290, with the CPU inside / within tests).
static V4 eval_premultiplied(const Scene& sc, const SceneBvh& bvh, V2 pt, V4 background) {
    std::vector<Fragment> frags;
    collect_fragments(sc, bvh, pt, nullptr, frags);
    float pr = background.x, pg = background.y, pb = background.z, pa = background.w;
    for (const Fragment& f : frags) {
        float br = pr * (1.0f - f.a) + f.r * f.a;
        float bg = pg * (1.0f - f.a) + f.g * f.a;
        float bb = pb * (1.0f - f.a) + f.b * f.a;
        float ba = pa * (1.0f - f.a) + f.a;
        pr = br;
        pg = bg;
        pb = bb;
        pa = ba;
    }
    return V4{pr, pg, pb, pa};
}

// ---------------------------------------------------------------- boundary sampling (backward/boundary.rs)
struct ShapeCdf {
    std::vector<size_t> shape_ids, group_ids;
    std::vector<float> cdf, pmf;
};
struct PathCdf {
    bool valid = false;
    std::vector<float> cdf, pmf;
    std::vector<size_t> point_id_map;
    float length = 0.0f;
};
static V2 bez2(V2 p0, V2 p1, V2 p2, float t) {
    float tt = 1.0f - t;
    return p0 * (tt * tt) + p1 * (2.0f * tt * t) + p2 * (t * t);
}
static V2 bez3(V2 p0, V2 p1, V2 p2, V2 p3, float t) {
    float tt = 1.0f - t;
    return p0 * (tt * tt * tt) + p1 * (3.0f * tt * tt * t) + p2 * (3.0f * tt * t * t) + p3 * (t * t * t);
}
static float segment_length_est(const PathG& p, size_t point_id, uint8_t nc, bool* ok) {  // boundary.rs:237-307
    V2 q0, q1, q2, q3;
    *ok = true;
    if (nc == 0) {
        if (!path_point(p, point_id, &q0) || !path_point(p, point_id + 1, &q1)) {
            *ok = false;
            return 0.0f;
        }
        return length(q1 - q0);
    }
    if (nc == 1) {
        if (!path_point(p, point_id, &q0) || !path_point(p, point_id + 1, &q1) || !path_point(p, point_id + 2, &q2)) {
            *ok = false;
            return 0.0f;
        }
        V2 v1 = bez2(q0, q1, q2, 0.5f);
        return length(v1 - q0) + length(q2 - v1);
    }
    if (nc == 2) {
        if (!path_point(p, point_id, &q0) || !path_point(p, point_id + 1, &q1) || !path_point(p, point_id + 2, &q2) ||
            !path_point(p, point_id + 3, &q3)) {
            *ok = false;
            return 0.0f;
        }
        V2 v1 = bez3(q0, q1, q2, q3, 1.0f / 3.0f);
        V2 v2 = bez3(q0, q1, q2, q3, 2.0f / 3.0f);
        return length(v1 - q0) + length(v2 - v1) + length(q3 - v2);
    }
    *ok = false;
    return 0.0f;
}
static float path_length(const PathG& p) {  // boundary.rs:230-309
    if (p.pts.empty()) return 0.0f;
    float len = 0.0f;
    size_t point_id = 0;
    for (uint8_t nc : p.ncp) {
        bool ok;
        float l = segment_length_est(p, point_id, nc, &ok);
        if (!ok) break;
        len += l;
        point_id += nc == 0 ? 1 : (nc == 1 ? 2 : 3);
    }
    return len;
}
static std::vector<float> compute_shape_lengths(const Scene& sc) {  // boundary.rs:200-227
    std::vector<float> out(sc.shapes.size(), 0.0f);
    for (size_t i = 0; i < sc.shapes.size(); ++i) {
        const Shape& s = sc.shapes[i];
        float l = 0.0f;
        if (s.kind == DVG_SHAPE_CIRCLE) {
            l = 2.0f * PI_F * std::fabs(s.prm[2]);
        } else if (s.kind == DVG_SHAPE_ELLIPSE) {
            float a = std::fabs(s.prm[2]), b = std::fabs(s.prm[3]);
            l = (a == 0.0f || b == 0.0f) ? 0.0f
                                         : PI_F * (3.0f * (a + b) - std::sqrt((3.0f * a + b) * (a + 3.0f * b)));
        } else if (s.kind == DVG_SHAPE_RECT) {
            float w = std::fabs(s.prm[2] - s.prm[0]), h = std::fabs(s.prm[3] - s.prm[1]);
            l = 2.0f * (w + h);
        } else if (s.kind == DVG_SHAPE_PATH) {
            l = path_length(s.path);
        }
        out[i] = l;
    }
    return out;
}
static bool build_shape_cdf(const Scene& sc, const std::vector<float>& lens, ShapeCdf* out) {  // boundary.rs:312-346
    float accum = 0.0f;
    for (size_t gi = 0; gi < sc.groups.size(); ++gi)
        for (size_t si : sc.groups[gi].shape_ids) {
            float l = si < lens.size() ? lens[si] : 0.0f;
            out->shape_ids.push_back(si);
            out->group_ids.push_back(gi);
            accum += l;
            out->cdf.push_back(accum);
            out->pmf.push_back(l);
        }
    if (accum <= 0.0f || !std::isfinite(accum) || out->cdf.empty()) return false;
    for (float& v : out->cdf) v /= accum;
    for (float& v : out->pmf) v /= accum;
    return true;
}
static std::vector<PathCdf> build_path_cdfs(const Scene& sc, const std::vector<float>& lens) {  // boundary.rs:349-451
    std::vector<PathCdf> out(sc.shapes.size());
    for (size_t si = 0; si < sc.shapes.size(); ++si) {
        const Shape& s = sc.shapes[si];
        if (s.kind != DVG_SHAPE_PATH) continue;
        float l = lens[si];
        if (l <= 0.0f || !std::isfinite(l)) continue;
        if (s.path.ncp.empty()) continue;
        float inv_length = 1.0f / l;
        PathCdf pc;
        size_t point_id = 0;
        for (uint8_t nc : s.path.ncp) {
            pc.point_id_map.push_back(point_id);
            bool ok;
            float seg_len = segment_length_est(s.path, point_id, nc, &ok);
            if (!ok) seg_len = 0.0f;
            if (nc == 0)
                point_id += 1;
            else if (nc == 1)
                point_id += 2;
            else if (nc == 2)
                point_id += 3;
            float seg_norm = seg_len * inv_length;
            pc.pmf.push_back(seg_norm);
            float acc = seg_norm + (pc.cdf.empty() ? 0.0f : pc.cdf.back());
            pc.cdf.push_back(acc);
        }
        pc.length = l;
        pc.valid = true;
        out[si] = pc;
    }
    return out;
}
static size_t sample_cdf(const std::vector<float>& cdf, float u, float* t_out) {  // boundary.rs:454-469
    if (cdf.empty()) {
        *t_out = 0.0f;
        return 0;
    }
    size_t idx = 0;
    while (idx < cdf.size() && u > cdf[idx]) idx += 1;
    if (idx >= cdf.size()) idx = cdf.size() - 1;
    float prev = idx == 0 ? 0.0f : cdf[idx - 1];
    float denom = std::fmax(cdf[idx] - prev, 1.0e-6f);
    *t_out = clampf((u - prev) / denom, 0.0f, 1.0f);
    return idx;
}
struct BData {
    size_t base_point_id = 0, point_id = 0;
    float t = 0.0f;
    bool is_stroke = false;
    bool join_cap = false;  // a join / cap edge sample (extension): t = (p - v) . n / r
};
// Share of a styled stroke's edge samples on its join and cap edges (extension).
const float kJoinCapShare = 0.25f;
static float len2f(float x, float y) { return std::sqrt(x * x + y * y); }
// The join and cap edges of a stroke with non-round joins or caps: the same sites,
// order and arithmetic as the library's kernel (sample_join_cap).
static V2 sample_join_cap(const Shape& s, float t, V2* normal, float* pdf, BData* data) {
    const PathG& path = s.path;
    const std::vector<SegData> segs = path_segments(s, s.stroke_width);
    const bool closed = path.closed;
    const int n = (int)segs.size();
    const int nj = s.join != DVG_JOIN_ROUND ? (closed ? n : n - 1) : 0;
    const int ncap = !closed && s.cap != DVG_CAP_ROUND ? 2 : 0;
    const int sites = nj + ncap;
    if (n <= 0 || sites <= 0) {
        *pdf = 0.0f;
        return mk(0, 0);
    }
    std::vector<size_t> seg_pid(n);
    for (int i = 0, pid = 0; i < n; ++i) {
        seg_pid[i] = (size_t)pid;
        pid += path.ncp[i] + 1;
    }
    int k = (int)(t * (float)sites);
    if (k > sites - 1) k = sites - 1;
    const float u = t * (float)sites - (float)k;
    *pdf /= (float)sites;
    V2 e[4], v = mk(0, 0), capdir = mk(0, 0);
    int ne = 0;
    size_t pid = 0;
    float r = 0.0f;
    if (k < nj) {
        const int vb = closed ? k : k + 1, va = vb > 0 ? vb - 1 : n - 1;
        v = segs[vb].p0;
        r = segs[vb].r0;
        pid = seg_pid[vb];
        V2 din = seg_dir1(segs[va]), dout = seg_dir0(segs[vb]);
        const float li = std::sqrt(din.x * din.x + din.y * din.y), lo = std::sqrt(dout.x * dout.x + dout.y * dout.y);
        if (!(li > 0.0f) || !(lo > 0.0f) || !(r > 0.0f)) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        din = mk(din.x / li, din.y / li);
        dout = mk(dout.x / lo, dout.y / lo);
        const float cr = cross2f(din.x, din.y, dout.x, dout.y);
        if (std::fabs(cr) < 1.0e-6f) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        const float sg = cr > 0.0f ? 1.0f : -1.0f;
        e[0] = mk(v.x + r * sg * din.y, v.y - r * sg * din.x);
        const V2 b = mk(v.x + r * sg * dout.y, v.y - r * sg * dout.x);
        ne = 1;
        if (s.join == DVG_JOIN_MITER) {
            const float sm = cross2f(b.x - e[0].x, b.y - e[0].y, dout.x, dout.y) / cr;
            const V2 m = mk(e[0].x + sm * din.x, e[0].y + sm * din.y);
            const float ml = std::sqrt((m.x - v.x) * (m.x - v.x) + (m.y - v.y) * (m.y - v.y));
            if (ml <= std::fmax(s.miter, 1.0f) * r) e[ne++] = m;
        }
        e[ne] = b;
    } else {
        const bool start = k == nj;
        const SegData& g = segs[start ? 0 : n - 1];
        V2 d;
        if (start) {
            const V2 d0 = seg_dir0(g);
            d = mk(-d0.x, -d0.y);
            v = g.p0;
            r = g.r0;
            pid = seg_pid[0];
        } else {
            d = seg_dir1(g);
            v = g.p3;
            r = g.r3;
            pid = path.pts.size() - 1;
        }
        const float l = std::sqrt(d.x * d.x + d.y * d.y);
        if (!(l > 0.0f) || !(r > 0.0f)) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        d = mk(d.x / l, d.y / l);
        capdir = d;
        const V2 np = mk(-d.y, d.x);
        e[0] = mk(v.x - r * np.x, v.y - r * np.y);
        if (s.cap == DVG_CAP_SQUARE) {
            e[1] = mk(e[0].x + r * d.x, e[0].y + r * d.y);
            e[2] = mk(v.x + r * np.x + r * d.x, v.y + r * np.y + r * d.y);
            e[3] = mk(v.x + r * np.x, v.y + r * np.y);
            ne = 3;
        } else {
            e[1] = mk(v.x + r * np.x, v.y + r * np.y);
            ne = 1;
        }
    }
    float len[3], total = 0.0f;
    for (int i = 0; i < ne; ++i) {
        len[i] = len2f(e[i + 1].x - e[i].x, e[i + 1].y - e[i].y);
        total += len[i];
    }
    if (!(total > 0.0f)) {
        *pdf = 0.0f;
        return mk(0, 0);
    }
    float sl = u * total;
    int i = 0;
    while (i < ne - 1 && sl > len[i]) sl -= len[i++];
    const float f = len[i] > 0.0f ? std::fmin(sl / len[i], 1.0f) : 0.0f;
    const V2 p = mk(e[i].x + f * (e[i + 1].x - e[i].x), e[i].y + f * (e[i + 1].y - e[i].y));
    const float ex = -(e[i + 1].y - e[i].y), ey = e[i + 1].x - e[i].x, el = len2f(ex, ey);
    V2 nn = el > 0.0f ? mk(ex / el, ey / el) : mk(0.0f, 0.0f);
    const float mx = 0.5f * (e[i].x + e[i + 1].x) - v.x, my = 0.5f * (e[i].y + e[i + 1].y) - v.y;
    const float side = (mx == 0.0f && my == 0.0f) ? nn.x * capdir.x + nn.y * capdir.y : nn.x * mx + nn.y * my;
    if (side < 0.0f) nn = mk(-nn.x, -nn.y);
    *pdf /= total;
    *normal = nn;
    (void)pid;
    data->join_cap = true;
    data->base_point_id = (size_t)k;  // the site
    data->point_id = (size_t)i;       // the edge of the site's polygon
    data->t = f;                      // the position along that edge
    return p;
}

// Forward-mode derivative of a join / cap site's polygon with respect to its vertex
// v, the control point q that sets the adjacent tangent(s) (qa before, qb after the
// vertex) and the radius: 7 partials (v.x, v.y, qa.x, qa.y, qb.x, qb.y, r).
struct Dl {
    float v;
    float d[7];
};
static Dl dl_const(float v) {
    Dl r;
    r.v = v;
    for (float& x : r.d) x = 0.0f;
    return r;
}
static Dl dl_var(float v, int k) {
    Dl r = dl_const(v);
    r.d[k] = 1.0f;
    return r;
}
static Dl operator+(const Dl& a, const Dl& b) {
    Dl r;
    r.v = a.v + b.v;
    for (int k = 0; k < 7; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
static Dl operator-(const Dl& a, const Dl& b) {
    Dl r;
    r.v = a.v - b.v;
    for (int k = 0; k < 7; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
static Dl operator*(const Dl& a, const Dl& b) {
    Dl r;
    r.v = a.v * b.v;
    for (int k = 0; k < 7; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
static Dl operator/(const Dl& a, const Dl& b) {
    Dl r;
    r.v = a.v / b.v;
    for (int k = 0; k < 7; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
static Dl dl_sqrt(const Dl& a) {
    Dl r;
    r.v = std::sqrt(a.v);
    for (int k = 0; k < 7; ++k) r.d[k] = r.v > 0.0f ? a.d[k] * (0.5f / r.v) : 0.0f;
    return r;
}
struct DV {
    Dl x, y;
};
static DV dv_add(const DV& a, const DV& b) { return DV{a.x + b.x, a.y + b.y}; }
static DV dv_sub(const DV& a, const DV& b) { return DV{a.x - b.x, a.y - b.y}; }
static DV dv_scale(const DV& a, const Dl& s) { return DV{a.x * s, a.y * s}; }
static DV dv_unit(const DV& a) {
    const Dl l = dl_sqrt(a.x * a.x + a.y * a.y);
    return DV{a.x / l, a.y / l};
}
// Point slot j of a path segment -> path point index (lines and quadratics repeat
// their last point; closed paths wrap).
static size_t seg_slot_point(const PathG& p, size_t pid, int nc, int j) {
    size_t idx = pid + (size_t)std::min(j, nc + 1);
    return p.closed ? idx % p.pts.size() : idx;
}
static int seg_dir0_slot(const SegData& g) {
    V2 d = g.p1 - g.p0;
    if (!(d.x == 0.0f && d.y == 0.0f)) return 1;
    d = g.p2 - g.p0;
    return !(d.x == 0.0f && d.y == 0.0f) ? 2 : 3;
}
static int seg_dir1_slot(const SegData& g) {
    V2 d = g.p3 - g.p2;
    if (!(d.x == 0.0f && d.y == 0.0f)) return 2;
    d = g.p3 - g.p1;
    return !(d.x == 0.0f && d.y == 0.0f) ? 1 : 0;
}
static V2 seg_slot(const SegData& g, int j) { return j == 0 ? g.p0 : j == 1 ? g.p1 : j == 2 ? g.p2 : g.p3; }
// Prefiltered stroke of a styled path (the library's extension; the crate's prefiltered
// stroke coverage is round, smoothstep(|d| + sw) - smoothstep(|d| - sw), sampling.rs:
// 240-260).  Where the closest point is a segment end that the point-sampled stroke
// excludes (end_excluded), the coverage is smoothstep(s + 2 sw) - smoothstep(s), s the
// signed distance (canvas space, negative inside) to the outer edges of that join or cap
// region, built in canvas space from the canvas images of the vertex and of the control
// points that set its tangents with the stroke width as radius: bevel edge; the two miter
// edges within the limit; a butt end's flat end; a square cap's three outer box edges.
// A reversal ends both bodies flat; a straight join (|cross| < 1e-6) keeps the round
// formula (returns false).  sd->d: partials with respect to (v, qa, qb) in canvas space
// and sw; ids: path points of v, qa, qb (-1: unused); q: their shape-space positions.
static bool styled_end_sd(const Group& grp, const Shape& s, size_t seg, float t, V2 pt, Dl* sd, long ids[3],
                          V2 q[3]) {
    if (s.kind != DVG_SHAPE_PATH || !(s.stroke_width > 0.0f)) return false;
    const PathG& path = s.path;
    const std::vector<SegData> segs = path_segments(s, s.stroke_width);
    const size_t n = segs.size();
    if (seg >= n || !end_excluded(s, seg, n, t)) return false;
    const bool closed = path.closed;
    std::vector<size_t> seg_pid(n);
    for (size_t i = 0, pid = 0; i < n; ++i) {
        seg_pid[i] = pid;
        pid += path.ncp[i] + 1;
    }
    auto canvas = [&](V2 p) { return xform_pt(grp.s2c, xform_pt(s.transform, p)); };
    ids[0] = ids[1] = ids[2] = -1;
    const bool at1 = t == 1.0f;
    const bool is_join = closed || (at1 ? seg + 1 < n : seg > 0);
    const Dl R = dl_var(s.stroke_width, 6);
    DV V, e[4];
    int ne = 1;
    bool fan = false, rect = false;
    if (is_join) {
        const size_t vb = at1 ? (seg + 1) % n : seg, va = vb > 0 ? vb - 1 : n - 1;
        const int sa = seg_dir1_slot(segs[va]), sb = seg_dir0_slot(segs[vb]);
        q[0] = segs[vb].p0;
        q[1] = seg_slot(segs[va], sa);
        q[2] = seg_slot(segs[vb], sb);
        ids[0] = (long)seg_pid[vb];
        ids[1] = (long)seg_slot_point(path, seg_pid[va], path.ncp[va], sa);
        ids[2] = (long)seg_slot_point(path, seg_pid[vb], path.ncp[vb], sb);
        const V2 vc = canvas(q[0]), ac = canvas(q[1]), bc = canvas(q[2]);
        if ((vc.x == ac.x && vc.y == ac.y) || (vc.x == bc.x && vc.y == bc.y)) return false;
        V = DV{dl_var(vc.x, 0), dl_var(vc.y, 1)};
        const DV QA{dl_var(ac.x, 2), dl_var(ac.y, 3)}, QB{dl_var(bc.x, 4), dl_var(bc.y, 5)};
        const DV din = dv_unit(dv_sub(V, QA)), dout = dv_unit(dv_sub(QB, V));
        const Dl cr = din.x * dout.y - din.y * dout.x;
        if (std::fabs(cr.v) < 1.0e-6f) {
            if (din.x.v * dout.x.v + din.y.v * dout.y.v > 0.0f) return false;
            const DV np{dl_const(0.0f) - din.y, din.x};
            e[0] = dv_sub(V, dv_scale(np, R));
            e[1] = dv_add(V, dv_scale(np, R));
        } else {
            const Dl sg = dl_const(cr.v > 0.0f ? 1.0f : -1.0f);
            e[0] = DV{V.x + R * sg * din.y, V.y - R * sg * din.x};
            const DV b{V.x + R * sg * dout.y, V.y - R * sg * dout.x};
            if (s.join == DVG_JOIN_MITER) {
                const Dl sm = ((b.x - e[0].x) * dout.y - (b.y - e[0].y) * dout.x) / cr;
                const DV m = dv_add(e[0], dv_scale(din, sm));
                const float ml = std::sqrt((m.x.v - vc.x) * (m.x.v - vc.x) + (m.y.v - vc.y) * (m.y.v - vc.y));
                if (ml <= std::fmax(s.miter, 1.0f) * R.v) e[ne++] = m;
            }
            e[ne] = b;
            fan = true;
        }
    } else {
        const bool start = !at1;
        const size_t sj = start ? 0 : n - 1;
        const SegData& g = segs[sj];
        const int sq = start ? seg_dir0_slot(g) : seg_dir1_slot(g);
        q[0] = start ? g.p0 : g.p3;
        q[start ? 2 : 1] = seg_slot(g, sq);
        ids[0] = (long)seg_slot_point(path, seg_pid[sj], path.ncp[sj], start ? 0 : 3);
        ids[start ? 2 : 1] = (long)seg_slot_point(path, seg_pid[sj], path.ncp[sj], sq);
        const V2 vc = canvas(q[0]), qc = canvas(q[start ? 2 : 1]);
        if (vc.x == qc.x && vc.y == qc.y) return false;
        V = DV{dl_var(vc.x, 0), dl_var(vc.y, 1)};
        const DV Q = start ? DV{dl_var(qc.x, 4), dl_var(qc.y, 5)} : DV{dl_var(qc.x, 2), dl_var(qc.y, 3)};
        const DV d = dv_unit(dv_sub(V, Q));
        const DV np{dl_const(0.0f) - d.y, d.x};
        e[0] = dv_sub(V, dv_scale(np, R));
        if (s.cap == DVG_CAP_SQUARE) {
            e[1] = dv_add(e[0], dv_scale(d, R));
            e[2] = dv_add(dv_add(V, dv_scale(np, R)), dv_scale(d, R));
            e[3] = dv_add(V, dv_scale(np, R));
            ne = 3;
            rect = true;
        } else {
            e[1] = dv_add(V, dv_scale(np, R));
        }
    }
    Dl best = dl_const(0.0f);
    for (int i = 0; i < ne; ++i) {
        const DV ex = dv_sub(e[i + 1], e[i]);
        const Dl ee = ex.x * ex.x + ex.y * ex.y;
        DV c = e[i];
        if (ee.v > 0.0f) {
            const Dl tt = ((dl_const(pt.x) - e[i].x) * ex.x + (dl_const(pt.y) - e[i].y) * ex.y) / ee;
            if (tt.v >= 1.0f)
                c = e[i + 1];
            else if (tt.v > 0.0f)
                c = dv_add(e[i], dv_scale(ex, tt));
        }
        const Dl dx = dl_const(pt.x) - c.x, dy = dl_const(pt.y) - c.y;
        const Dl d2 = dx * dx + dy * dy;
        if (i == 0 || d2.v < best.v) best = d2;
    }
    const Dl dist = dl_sqrt(best);
    auto val = [](const DV& a) { return mk(a.x.v, a.y.v); };
    bool inside = false;
    if (fan)
        for (int i = 0; i < ne; ++i) inside = inside || in_triangle(pt, val(V), val(e[i]), val(e[i + 1]));
    if (rect) inside = in_triangle(pt, val(e[0]), val(e[1]), val(e[2])) || in_triangle(pt, val(e[0]), val(e[2]), val(e[3]));
    *sd = inside ? dl_const(0.0f) - dist : dist;
    return true;
}
static bool styled_end_value(const Group& grp, const Shape& s, size_t seg, float t, V2 pt, float* sd) {
    Dl d;
    long ids[3];
    V2 q[3];
    if (!styled_end_sd(grp, s, seg, t, pt, &d, ids, q)) return false;
    *sd = d.v;
    return true;
}
// Adjoint of styled_end_sd: d_s times its partials through the shape and group
// transforms into the path points and both transforms; returns d_pt (the region moves
// with its three points, so d/dpt = -(the sum of their partials)).
static V2 d_styled_end(const Group& grp, size_t group_id, const Shape& s, size_t shape_id, const Dl& sd, float d_s,
                       const long ids[3], const V2 q[3], Grads& g) {
    M3 d_s2c = zero3(), d_st = zero3();
    V2 sum = mk(0, 0);
    for (int j = 0; j < 3; ++j) {
        if (ids[j] < 0) continue;
        const V2 gc = mk(d_s * sd.d[2 * j], d_s * sd.d[2 * j + 1]);
        sum = sum + gc;
        const V2 qg = xform_pt(s.transform, q[j]);
        V2 g_qg = mk(0, 0), g_q = mk(0, 0);
        d_xform_pt(grp.s2c, qg, gc, &d_s2c, &g_qg);
        d_xform_pt(s.transform, q[j], g_qg, &d_st, &g_q);
        g.points[2 * (s.path.point_base + (size_t)ids[j])] += g_q.x;
        g.points[2 * (s.path.point_base + (size_t)ids[j]) + 1] += g_q.y;
    }
    add_group_transform(g, group_id, d_s2c);
    add_shape_transform(g, shape_id, d_st);
    return sum * -1.0f;
}
// The styled prefiltered stroke's adjoint for d_s = dL/ds: geometry and transforms into
// g, the stroke-width part of ds/dsw * d_s into *d_sw, dL/dpt into *d_pt.
static bool styled_end_backward(const Group& grp, size_t group_id, const Shape& s, size_t shape_id, size_t seg, float t,
                                V2 pt, float d_s, Grads& g, float* d_sw, V2* d_pt) {
    Dl sd;
    long ids[3];
    V2 q[3];
    if (!styled_end_sd(grp, s, seg, t, pt, &sd, ids, q)) return false;
    *d_sw = d_s * sd.d[6];
    *d_pt = d_styled_end(grp, group_id, s, shape_id, sd, d_s, ids, q, g);
    return true;
}
// Normal velocity of the edge point sampled at (site, edge, f): w[k] = dp/dtheta_k . n
// for theta = (v, qa, qb, r); ids = path points of v, qa, qb (-1: not used).
static bool join_cap_velocity(const Shape& s, size_t site, size_t edge, float f, V2 n, float w[7], long ids[3]) {
    const PathG& path = s.path;
    const std::vector<SegData> segs = path_segments(s, s.stroke_width);
    const bool closed = path.closed;
    const int nseg = (int)segs.size();
    const int nj = s.join != DVG_JOIN_ROUND ? (closed ? nseg : nseg - 1) : 0;
    std::vector<size_t> seg_pid(nseg);
    for (int i = 0, pid = 0; i < nseg; ++i) {
        seg_pid[i] = (size_t)pid;
        pid += path.ncp[i] + 1;
    }
    const int k = (int)site;
    ids[0] = ids[1] = ids[2] = -1;
    DV e[4];
    int ne = 0;
    if (k < nj) {
        const int vb = closed ? k : k + 1, va = vb > 0 ? vb - 1 : nseg - 1;
        const int sa = seg_dir1_slot(segs[va]), sb = seg_dir0_slot(segs[vb]);
        const V2 v = segs[vb].p0, qa = seg_slot(segs[va], sa), qb = seg_slot(segs[vb], sb);
        ids[0] = (long)seg_pid[vb];
        ids[1] = (long)seg_slot_point(path, seg_pid[va], path.ncp[va], sa);
        ids[2] = (long)seg_slot_point(path, seg_pid[vb], path.ncp[vb], sb);
        const DV V{dl_var(v.x, 0), dl_var(v.y, 1)}, QA{dl_var(qa.x, 2), dl_var(qa.y, 3)},
            QB{dl_var(qb.x, 4), dl_var(qb.y, 5)};
        const Dl R = dl_var(segs[vb].r0, 6);
        const DV din = dv_unit(dv_sub(V, QA)), dout = dv_unit(dv_sub(QB, V));
        const Dl cr = din.x * dout.y - din.y * dout.x;
        if (std::fabs(cr.v) < 1.0e-6f) return false;
        const Dl sg = dl_const(cr.v > 0.0f ? 1.0f : -1.0f);
        e[0] = DV{V.x + R * sg * din.y, V.y - R * sg * din.x};
        const DV b{V.x + R * sg * dout.y, V.y - R * sg * dout.x};
        ne = 1;
        if (s.join == DVG_JOIN_MITER) {
            const Dl sm = ((b.x - e[0].x) * dout.y - (b.y - e[0].y) * dout.x) / cr;
            const DV m = dv_add(e[0], dv_scale(din, sm));
            const float ml = std::sqrt((m.x.v - v.x) * (m.x.v - v.x) + (m.y.v - v.y) * (m.y.v - v.y));
            if (ml <= std::fmax(s.miter, 1.0f) * R.v) e[ne++] = m;
        }
        e[ne] = b;
    } else {
        const bool start = k == nj;
        const int si = start ? 0 : nseg - 1;
        const SegData& g = segs[si];
        const int sq = start ? seg_dir0_slot(g) : seg_dir1_slot(g);
        const V2 v = start ? g.p0 : g.p3, q = seg_slot(g, sq);
        ids[0] = (long)(start ? seg_pid[0] : path.pts.size() - 1);
        ids[start ? 2 : 1] = (long)seg_slot_point(path, seg_pid[si], path.ncp[si], sq);
        const DV V{dl_var(v.x, 0), dl_var(v.y, 1)};
        const DV Q = start ? DV{dl_var(q.x, 4), dl_var(q.y, 5)} : DV{dl_var(q.x, 2), dl_var(q.y, 3)};
        const Dl R = dl_var(start ? g.r0 : g.r3, 6);
        const DV d = start ? dv_unit(dv_sub(V, Q)) : dv_unit(dv_sub(V, Q));  // outward along the end
        const DV np{dl_const(0.0f) - d.y, d.x};
        e[0] = dv_sub(V, dv_scale(np, R));
        if (s.cap == DVG_CAP_SQUARE) {
            e[1] = dv_add(e[0], dv_scale(d, R));
            e[2] = dv_add(dv_add(V, dv_scale(np, R)), dv_scale(d, R));
            e[3] = dv_add(V, dv_scale(np, R));
            ne = 3;
        } else {
            e[1] = dv_add(V, dv_scale(np, R));
            ne = 1;
        }
    }
    if ((int)edge >= ne) return false;
    const DV& a = e[edge];
    const DV& b = e[edge + 1];
    const Dl F = dl_const(f);
    const DV p = dv_add(a, dv_scale(dv_sub(b, a), F));
    for (int j = 0; j < 7; ++j) w[j] = p.x.d[j] * n.x + p.y.d[j] * n.y;
    return true;
}
static V2 sample_boundary_path(const PathG& path, const PathCdf& pc, float path_len, float t, V2* normal, float* pdf,
                               BData* data, float stroke_direction, float stroke_radius,
                               const Shape* style) {  // boundary.rs:630-842
    size_t num_points = path.pts.size();
    size_t num_base = path.ncp.size();
    if (num_points == 0 || num_base == 0) {
        *pdf = 0.0f;
        return mk(0, 0);
    }
    const bool styled = stroke_direction != 0.0f && style && style_nonround(*style);
    if (styled) {  // extension: a share of the samples on the join / cap edges (both sides draw them)
        const float q = kJoinCapShare;
        if (t < q) {
            *pdf *= 2.0f * q;
            return sample_join_cap(*style, t / q, normal, pdf, data);
        }
        t = (t - q) / (1.0f - q);
        *pdf *= 1.0f - q;
    }
    if (stroke_direction != 0.0f && !path.closed && (!styled || style->cap == DVG_CAP_ROUND)) {
        float cap_length = 0.0f;
        if (path.has_thick) {
            if (!path.thick.empty()) cap_length = PI_F * (path.thick[0] + path.thick.back());
        } else {
            cap_length = 2.0f * PI_F * stroke_radius;
        }
        float denom = cap_length + path_len;
        if (denom > 0.0f) {
            float cap_prob = cap_length / denom;
            if (t < cap_prob) {
                t /= cap_prob;
                *pdf *= cap_prob;
                float r0 = stroke_radius, r1 = stroke_radius;
                if (path.has_thick && !path.thick.empty()) {
                    r0 = path.thick[0];
                    r1 = path.thick.back();
                }
                float angle = 2.0f * PI_F * t;
                if (stroke_direction < 0.0f) {
                    V2 p0 = path.pts[0];
                    V2 off = mk(r0 * std::cos(angle), r0 * std::sin(angle));
                    *normal = normalize(off);
                    *pdf /= 2.0f * PI_F * r0;
                    data->base_point_id = 0;
                    data->point_id = 0;
                    data->t = 0.0f;
                    return p0 + off;
                } else {
                    V2 p0 = path.pts[num_points - 1];
                    V2 off = mk(r1 * std::cos(angle), r1 * std::sin(angle));
                    *normal = normalize(off);
                    *pdf /= 2.0f * PI_F * r1;
                    data->base_point_id = num_base - 1;
                    size_t controls = path.ncp[data->base_point_id];
                    data->point_id = num_points >= 2 + controls ? num_points - (2 + controls) : 0;
                    data->t = 1.0f;
                    return p0 + off;
                }
            } else {
                t = (t - cap_prob) / (1.0f - cap_prob);
                *pdf *= 1.0f - cap_prob;
            }
        }
    }
    float local_t;
    size_t sample_id = sample_cdf(pc.cdf, t, &local_t);
    if (sample_id >= pc.point_id_map.size()) {
        *pdf = 0.0f;
        return mk(0, 0);
    }
    size_t point_id = pc.point_id_map[sample_id];
    data->base_point_id = sample_id;
    data->point_id = point_id;
    data->t = local_t;
    if (local_t < -1.0e-3f || local_t > 1.0f + 1.0e-3f) {
        *pdf = 0.0f;
        return mk(0, 0);
    }
    auto next_index = [&](size_t idx) -> size_t {
        if (path.closed) return idx % num_points;
        return std::min(idx, num_points >= 1 ? num_points - 1 : 0);
    };
    uint8_t nc = sample_id < path.ncp.size() ? path.ncp[sample_id] : 0;
    float pmf = sample_id < pc.pmf.size() ? pc.pmf[sample_id] : 0.0f;
    V2 q[4];
    float r[4];
    if (nc == 0) {
        if (!path_point_radius(path, point_id, stroke_radius, &q[0], &r[0]) ||
            !path_point_radius(path, next_index(point_id + 1), stroke_radius, &q[1], &r[1])) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        V2 tangent = q[1] - q[0];
        float tan_len = length(tangent);
        if (tan_len == 0.0f) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        *normal = mk(-tangent.y, tangent.x) / tan_len;
        *pdf *= pmf / tan_len;
        V2 out = q[0] + tangent * local_t;
        if (stroke_direction != 0.0f) {
            float rr = r[0] + local_t * (r[1] - r[0]);
            out += *normal * (stroke_direction * rr);
            if (stroke_direction < 0.0f) *normal = *normal * -1.0f;
        }
        return out;
    }
    if (nc == 1) {
        if (!path_point_radius(path, point_id, stroke_radius, &q[0], &r[0]) ||
            !path_point_radius(path, point_id + 1, stroke_radius, &q[1], &r[1]) ||
            !path_point_radius(path, next_index(point_id + 2), stroke_radius, &q[2], &r[2])) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        float tt = 1.0f - local_t;
        V2 ev = q[0] * (tt * tt) + q[1] * (2.0f * tt * local_t) + q[2] * (local_t * local_t);
        V2 tangent = (q[1] - q[0]) * (2.0f * tt) + (q[2] - q[1]) * (2.0f * local_t);
        float tan_len = length(tangent);
        if (tan_len == 0.0f) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        *normal = mk(-tangent.y, tangent.x) / tan_len;
        *pdf *= pmf / tan_len;
        V2 out = ev;
        if (stroke_direction != 0.0f) {
            float rr = r[0] * (tt * tt) + r[1] * (2.0f * tt * local_t) + r[2] * (local_t * local_t);
            out += *normal * (stroke_direction * rr);
            if (stroke_direction < 0.0f) *normal = *normal * -1.0f;
        }
        return out;
    }
    if (nc == 2) {
        if (!path_point_radius(path, point_id, stroke_radius, &q[0], &r[0]) ||
            !path_point_radius(path, point_id + 1, stroke_radius, &q[1], &r[1]) ||
            !path_point_radius(path, point_id + 2, stroke_radius, &q[2], &r[2]) ||
            !path_point_radius(path, next_index(point_id + 3), stroke_radius, &q[3], &r[3])) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        float tt = 1.0f - local_t;
        V2 ev = q[0] * (tt * tt * tt) + q[1] * (3.0f * tt * tt * local_t) + q[2] * (3.0f * tt * local_t * local_t) +
                q[3] * (local_t * local_t * local_t);
        V2 tangent = (q[1] - q[0]) * (3.0f * tt * tt) + (q[2] - q[1]) * (6.0f * tt * local_t) +
                     (q[3] - q[2]) * (3.0f * local_t * local_t);
        float tan_len = length(tangent);
        if (tan_len == 0.0f) {
            *pdf = 0.0f;
            return mk(0, 0);
        }
        *normal = mk(-tangent.y, tangent.x) / tan_len;
        *pdf *= pmf / tan_len;
        V2 out = ev;
        if (stroke_direction != 0.0f) {
            float rr = r[0] * (tt * tt * tt) + r[1] * (3.0f * tt * tt * local_t) +
                       r[2] * (3.0f * tt * local_t * local_t) + r[3] * (local_t * local_t * local_t);
            out += *normal * (stroke_direction * rr);
            if (stroke_direction < 0.0f) *normal = *normal * -1.0f;
        }
        return out;
    }
    *pdf = 0.0f;
    return mk(0, 0);
}
static bool sample_boundary_point(const Scene& sc, size_t shape_id, size_t group_id, float t, float shape_length,
                                  const PathCdf* pc, V2* pt_out, V2* normal_out, float* pdf_out,
                                  BData* data) {  // boundary.rs:472-627
    if (group_id >= sc.groups.size() || shape_id >= sc.shapes.size()) return false;
    const Group& g = sc.groups[group_id];
    const Shape& s = sc.shapes[shape_id];
    if (g.fill < 0 && g.stroke < 0) return false;
    float pdf = 1.0f;
    float local_t = t;
    bool stroke_perturb = false;
    if (g.fill >= 0 && g.stroke >= 0) {
        if (local_t < 0.5f) {
            stroke_perturb = false;
            local_t *= 2.0f;
            pdf = 0.5f;
        } else {
            stroke_perturb = true;
            local_t = 2.0f * (local_t - 0.5f);
            pdf = 0.5f;
        }
    } else if (g.stroke >= 0) {
        stroke_perturb = true;
    }
    float stroke_direction = 0.0f;
    if (stroke_perturb) {
        if (local_t < 0.5f) {
            stroke_direction = -1.0f;
            local_t *= 2.0f;
            pdf *= 0.5f;
        } else {
            stroke_direction = 1.0f;
            local_t = 2.0f * (local_t - 0.5f);
            pdf *= 0.5f;
        }
    }
    *data = BData();
    data->is_stroke = stroke_perturb;
    V2 normal = mk(0, 0);
    V2 pt;
    if (s.kind == DVG_SHAPE_CIRCLE) {
        float r = std::fabs(s.prm[2]);
        if (r <= 0.0f) return false;
        float angle = 2.0f * PI_F * local_t;
        V2 off = mk(r * std::cos(angle), r * std::sin(angle));
        normal = normalize(off);
        pdf /= 2.0f * PI_F * r;
        V2 out = mk(s.prm[0], s.prm[1]) + off;
        if (stroke_direction != 0.0f) {
            out += normal * (stroke_direction * s.stroke_width);
            if (stroke_direction < 0.0f) normal = normal * -1.0f;
        }
        pt = out;
    } else if (s.kind == DVG_SHAPE_ELLIPSE) {
        float rx = std::fabs(s.prm[2]), ry = std::fabs(s.prm[3]);
        if (rx <= 0.0f || ry <= 0.0f) return false;
        float angle = 2.0f * PI_F * local_t;
        float sn = std::sin(angle), cs = std::cos(angle);
        V2 off = mk(rx * cs, ry * sn);
        float dxdt = -rx * sn * 2.0f * PI_F;
        float dydt = ry * cs * 2.0f * PI_F;
        normal = normalize(mk(dydt, -dxdt));
        pdf /= std::sqrt(dxdt * dxdt + dydt * dydt);
        V2 out = mk(s.prm[0], s.prm[1]) + off;
        if (stroke_direction != 0.0f) {
            out += normal * (stroke_direction * s.stroke_width);
            if (stroke_direction < 0.0f) normal = normal * -1.0f;
        }
        pt = out;
    } else if (s.kind == DVG_SHAPE_RECT) {
        V2 mn = mk(s.prm[0], s.prm[1]), mx = mk(s.prm[2], s.prm[3]);
        float w = mx.x - mn.x, h = mx.y - mn.y;
        if (w == 0.0f && h == 0.0f) return false;
        pdf /= 2.0f * (w + h);
        V2 out = mk(0, 0);
        if (local_t <= w / (w + h)) {
            local_t *= (w + h) / w;
            if (local_t < 0.5f) {
                normal = mk(0.0f, -1.0f);
                out = mn + mk(2.0f * local_t * (mx.x - mn.x), 0.0f);
            } else {
                normal = mk(0.0f, 1.0f);
                out = mk(mn.x, mx.y) + mk(2.0f * (local_t - 0.5f) * (mx.x - mn.x), 0.0f);
            }
        } else {
            local_t = (local_t - w / (w + h)) * (w + h) / h;
            if (local_t < 0.5f) {
                normal = mk(-1.0f, 0.0f);
                out = mn + mk(0.0f, 2.0f * local_t * (mx.y - mn.y));
            } else {
                normal = mk(1.0f, 0.0f);
                out = mk(mx.x, mn.y) + mk(0.0f, 2.0f * (local_t - 0.5f) * (mx.y - mn.y));
            }
        }
        if (stroke_direction != 0.0f) {
            out += normal * (stroke_direction * s.stroke_width);
            if (stroke_direction < 0.0f) normal = normal * -1.0f;
        }
        pt = out;
    } else if (s.kind == DVG_SHAPE_PATH) {
        if (!pc || !pc->valid) return false;
        if (pc->length <= 0.0f) return false;
        pt = sample_boundary_path(s.path, *pc, shape_length, local_t, &normal, &pdf, data, stroke_direction,
                                  s.stroke_width, &s);
    } else {
        return false;
    }
    if (!std::isfinite(pdf) || pdf <= 0.0f) return false;
    *pt_out = pt;
    *normal_out = normal;
    *pdf_out = pdf;
    return true;
}
static void accumulate_boundary_gradient(const Shape& s, size_t shape_id, float contrib, float t, V2 normal,
                                         const BData& bd, Grads& g, const M3& group_s2c, V2 local_pt,
                                         size_t group_id) {  // boundary.rs:970-1148
    if (!std::isfinite(contrib)) return;
    const PathG& path = s.path;
    size_t pbase = path.point_base;
    if (bd.join_cap) {  // extension: exact normal velocity of a join / cap edge point
        float w[7];
        long ids[3];
        if (join_cap_velocity(s, bd.base_point_id, bd.point_id, bd.t, normal, w, ids)) {
            for (int j = 0; j < 3; ++j)
                if (ids[j] >= 0) {
                    g.points[2 * (pbase + (size_t)ids[j])] += w[2 * j] * contrib;
                    g.points[2 * (pbase + (size_t)ids[j]) + 1] += w[2 * j + 1] * contrib;
                }
            if (path.has_thick)
                g.thickness[pbase + (size_t)ids[0]] += w[6] * contrib;
            else
                g.stroke_width[shape_id] += w[6] * contrib;
        }
    } else if (bd.is_stroke) {
        bool has_thick = s.kind == DVG_SHAPE_PATH && path.has_thick;
        if (has_thick) {
            size_t n = path.thick.size();
            auto addt = [&](size_t i, float v) {
                if (i < n) g.thickness[pbase + i] += v;
            };
            size_t pid = bd.point_id;
            float t2 = bd.t;
            uint8_t nc = bd.base_point_id < path.ncp.size() ? path.ncp[bd.base_point_id] : 0;
            size_t np = path.pts.size();
            if (nc == 0) {
                size_t i1 = path.closed ? (pid + 1) % np : pid + 1;
                addt(pid, (1.0f - t2) * contrib);
                addt(i1, t2 * contrib);
            } else if (nc == 1) {
                size_t i2 = path.closed ? (pid + 2) % np : pid + 2;
                float tt = 1.0f - t2;
                addt(pid, tt * tt * contrib);
                addt(pid + 1, 2.0f * tt * t2 * contrib);
                addt(i2, t2 * t2 * contrib);
            } else if (nc == 2) {
                size_t i3 = path.closed ? (pid + 3) % np : pid + 3;
                float tt = 1.0f - t2;
                addt(pid, tt * tt * tt * contrib);
                addt(pid + 1, 3.0f * tt * tt * t2 * contrib);
                addt(pid + 2, 3.0f * tt * t2 * t2 * contrib);
                addt(i3, t2 * t2 * t2 * contrib);
            }
        } else {
            g.stroke_width[shape_id] += contrib;
        }
    }
    float* dp = &g.shape_params[4 * shape_id];
    if (s.kind == DVG_SHAPE_CIRCLE) {
        dp[0] += normal.x * contrib;
        dp[1] += normal.y * contrib;
        dp[2] += contrib;
    } else if (s.kind == DVG_SHAPE_ELLIPSE) {
        dp[0] += normal.x * contrib;
        dp[1] += normal.y * contrib;
        float angle = 2.0f * PI_F * t;
        dp[2] += std::cos(angle) * normal.x * contrib;
        dp[3] += std::sin(angle) * normal.y * contrib;
    } else if (s.kind == DVG_SHAPE_PATH && !bd.join_cap) {
        size_t np = path.pts.size();
        auto add_point = [&](size_t idx, float w) {
            size_t index = path.closed ? idx % np : idx;
            if (index < np) {
                g.points[2 * (pbase + index)] += normal.x * (w * contrib);
                g.points[2 * (pbase + index) + 1] += normal.y * (w * contrib);
            }
        };
        size_t pid = bd.point_id;
        float t2 = bd.t;
        uint8_t nc = bd.base_point_id < path.ncp.size() ? path.ncp[bd.base_point_id] : 0;
        if (nc == 0) {
            add_point(pid, 1.0f - t2);
            add_point(pid + 1, t2);
        } else if (nc == 1) {
            float tt = 1.0f - t2;
            add_point(pid, tt * tt);
            add_point(pid + 1, 2.0f * tt * t2);
            add_point(pid + 2, t2 * t2);
        } else if (nc == 2) {
            float tt = 1.0f - t2;
            add_point(pid, tt * tt * tt);
            add_point(pid + 1, 3.0f * tt * tt * t2);
            add_point(pid + 2, 3.0f * tt * t2 * t2);
            add_point(pid + 3, t2 * t2 * t2);
        }
    } else if (s.kind == DVG_SHAPE_RECT) {
        if (normal == mk(-1.0f, 0.0f))
            dp[0] += -contrib;
        else if (normal == mk(1.0f, 0.0f))
            dp[2] += contrib;
        else if (normal == mk(0.0f, -1.0f))
            dp[1] += -contrib;
        else if (normal == mk(0.0f, 1.0f))
            dp[3] += contrib;
    }
    M3 s2c = mul3(group_s2c, s.transform);
    M3 d_s2c = zero3();
    V2 d_lp = mk(0, 0);
    d_xform_pt(s2c, local_pt, normal * contrib, &d_s2c, &d_lp);
    M3 d_group = mul3(d_s2c, transpose3(s.transform));
    M3 d_shape = mul3(transpose3(group_s2c), d_s2c);
    float* dg = &g.group_transform[9 * group_id];
    float* ds = &g.shape_transform[9 * shape_id];
    for (int i = 0; i < 9; ++i) {
        dg[i] = dg[i] + d_group.m[i / 3][i % 3];
        ds[i] = ds[i] + d_shape.m[i / 3][i % 3];
    }
}
struct BoundaryTables {
    std::vector<float> lens;
    ShapeCdf cdf;
    bool ok = false;
    std::vector<PathCdf> path_cdfs;
};
static BoundaryTables build_boundary_tables(const Scene& sc) {
    BoundaryTables bt;
    if (sc.groups.empty()) return bt;
    bt.lens = compute_shape_lengths(sc);
    bt.ok = build_shape_cdf(sc, bt.lens, &bt.cdf);
    bt.path_cdfs = build_path_cdfs(sc, bt.lens);
    return bt;
}
// One boundary sample (boundary.rs:141-196 + render_edge_sample 845-967).
// pdf_scale: boundary samples drawn / W*H*spp.  The crate always draws W*H*spp and its
// edge term carries no 1/N (the weight image and the normalised coordinates hold it),
// so another sample count rescales every sample's pdf to keep the same expectation
// (exactly 1 for the crate's count).
//
// boundary_eval is the part after the two draws: the edge term of the boundary point at
// parameter t of shape-cdf entry sample_id.  Its contribution is multiplied by `weight`
// (1 for a drawn sample) and its colours are taken `offset` (normalised canvas units; the
// crate's 1e-4) either side of the point along the canvas normal.
static void boundary_eval(const Scene& sc, const SceneBvh& bvh, const BoundaryTables& bt, size_t sample_id, float t,
                          const float* d_render, const std::vector<float>& wimg, Grads& g, bool compute_translation,
                          float pdf_scale, float weight, float offset) {
    if (sample_id >= bt.cdf.shape_ids.size()) return;
    size_t shape_id = bt.cdf.shape_ids[sample_id];
    size_t group_id = bt.cdf.group_ids[sample_id];
    float shape_pmf = sample_id < bt.cdf.pmf.size() ? bt.cdf.pmf[sample_id] : 0.0f;
    if (shape_pmf <= 0.0f) return;
    float shape_length = shape_id < bt.lens.size() ? bt.lens[shape_id] : 0.0f;
    const PathCdf* pc = shape_id < bt.path_cdfs.size() ? &bt.path_cdfs[shape_id] : nullptr;
    V2 local_pt, normal;
    float bpdf;
    BData data;
    if (!sample_boundary_point(sc, shape_id, group_id, t, shape_length, pc, &local_pt, &normal, &bpdf, &data)) return;
    if (bpdf <= 0.0f) return;
    const Group& grp = sc.groups[group_id];
    const Shape& shp = sc.shapes[shape_id];
    M3 s2c = mul3(grp.s2c, shp.transform);
    V2 bpt = xform_pt(s2c, local_pt);
    M3 shape_inv;
    if (!inverse3(shp.transform, &shape_inv)) shape_inv = identity3();
    M3 composite_inv = mul3(shape_inv, grp.c2s);
    V2 normal_canvas = xform_normal(composite_inv, normal);
    bpt.x /= (float)sc.w;
    bpt.y /= (float)sc.h;
    float pdf = shape_pmf * bpdf * pdf_scale;
    // render_edge_sample
    int width = (int)sc.w, height = (int)sc.h;
    if (width <= 0 || height <= 0) return;
    if (pdf <= 0.0f) return;
    int bx = to_i32(bpt.x * (float)width), by = to_i32(bpt.y * (float)height);
    if (bx < 0 || bx >= width || by < 0 || by >= height) return;
    size_t pixel_index = (size_t)by * width + bx;
    V4 bg = sample_background(sc, pixel_index);
    EdgeQuery iq{group_id, shape_id, false}, oq{group_id, shape_id, false};
    V2 n = normal_canvas;
    V4 ci = sample_color(sc, bvh, bpt - n * offset, &bg, nullptr, &iq, nullptr, -1, pixel_index);
    V4 co = sample_color(sc, bvh, bpt + n * offset, &bg, nullptr, &oq, nullptr, -1, pixel_index);
    if (!iq.hit && !oq.hit) return;
    if (!iq.hit) {
        n = n * -1.0f;
        std::swap(ci, co);
    }
    V2 sbp = mk(bpt.x * (float)width, bpt.y * (float)height);
    V4 dc = gather_d_color(sc, d_render, wimg, sbp);
    float norm = (float)sc.w * (float)sc.h;
    if (norm > 0.0f) {
        dc.x /= norm;
        dc.y /= norm;
        dc.z /= norm;
        dc.w /= norm;
    }
    V4 diff{ci.x - co.x, ci.y - co.y, ci.z - co.z, ci.w - co.w};
    float contrib = dot4(diff, dc) / pdf;
    if (!std::isfinite(contrib)) return;
    contrib *= weight;
    accumulate_boundary_gradient(shp, shape_id, contrib, t, n, data, g, grp.s2c, local_pt, group_id);
    if (compute_translation && g.has_translation) {
        size_t ti = pixel_index * 2;
        if (ti + 1 < g.translation.size()) {
            g.translation[ti] += n.x * contrib;
            g.translation[ti + 1] += n.y * contrib;
        }
    }
}

static void boundary_sample(const Scene& sc, const SceneBvh& bvh, const BoundaryTables& bt, uint64_t idx,
                            uint32_t rng_kind, uint32_t seed, const float* d_render, const std::vector<float>& wimg,
                            Grads& g, bool compute_translation, float pdf_scale) {
    float u, t;
    boundary_rng(rng_kind, idx, seed, &u, &t);
    float dummy;
    size_t sample_id = sample_cdf(bt.cdf.cdf, u, &dummy);
    boundary_eval(sc, bvh, bt, sample_id, t, d_render, wimg, g, compute_translation, pdf_scale, 1.0f, 1.0e-4f);
}

// Interior sample (render.rs:95-169).
static void interior_sample(const Scene& sc, const SceneBvh& bvh, const SampleSpec& sp, uint64_t idx,
                            const float* d_render, const std::vector<float>& wimg, Grads& g, bool translation) {
    V2 pt;
    size_t pixel_index;
    sample_position(sc, sp, idx, &pt, &pixel_index);
    V2 npt = mk(pt.x / (float)sc.w, pt.y / (float)sc.h);
    V4 bg = sample_background(sc, pixel_index);
    V4 dcol = gather_d_color(sc, d_render, wimg, pt);
    V4 color = sp.prefilter
                   ? sample_color_prefiltered(sc, bvh, npt, &bg, &dcol, &g, translation ? (long)pixel_index : -1,
                                              pixel_index)
                   : sample_color(sc, bvh, npt, &bg, &dcol, nullptr, &g, translation ? (long)pixel_index : -1,
                                  pixel_index);
    accumulate_filter_gradient(sc, color, d_render, wimg, pt, &g.filter_radius);
}

static void export_grads(const Grads& g, dvg_grads* out, const dvg_scene_desc* d) {
    auto cp = [](float* dst, const std::vector<float>& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(float));
    };
    cp(out->d_shape_params, g.shape_params);
    cp(out->d_shape_transform, g.shape_transform);
    cp(out->d_shape_stroke_width, g.stroke_width);
    cp(out->d_points, g.points);
    cp(out->d_thickness, g.thickness);
    cp(out->d_group_transform, g.group_transform);
    cp(out->d_paint_params, g.paint_params);
    cp(out->d_stop_offsets, g.stop_offsets);
    cp(out->d_stop_colors, g.stop_colors);
    if (out->d_filter_radius) out->d_filter_radius[0] = g.filter_radius;
    if (out->d_background)
        for (int i = 0; i < 4; ++i) out->d_background[i] = g.background[i];
    if (out->d_background_image) {
        if (g.has_bg_image)
            cp(out->d_background_image, g.bg_image);
        else
            std::memset(out->d_background_image, 0, (size_t)d->width * d->height * 4 * sizeof(float));
    }
    if (out->d_translation) {
        if (g.has_translation)
            cp(out->d_translation, g.translation);
        else
            std::memset(out->d_translation, 0, (size_t)d->width * d->height * 2 * sizeof(float));
    }
}

template <typename F>
static void parallel_for(uint64_t begin, uint64_t end, int threads, F&& body) {
    if (threads <= 1 || end - begin < 1024) {
        body(0, begin, end);
        return;
    }
    std::vector<std::thread> pool;
    uint64_t n = end - begin;
    for (int t = 0; t < threads; ++t) {
        uint64_t b = begin + n * t / threads, e = begin + n * (t + 1) / threads;
        pool.emplace_back([&, t, b, e]() { body(t, b, e); });
    }
    for (auto& th : pool) th.join();
}

}  // namespace orc

using namespace orc;

static SampleSpec make_spec(const dvg_render_options* o) {
    SampleSpec sp;
    sp.sx_n = o->samples_x > 0 ? o->samples_x : 1;
    sp.sy_n = o->samples_y > 0 ? o->samples_y : 1;
    sp.prefilter = o->use_prefiltering != 0;
    sp.jitter = o->jitter != 0 && !sp.prefilter;
    sp.seed = o->seed;
    return sp;
}

extern "C" int oracle_weight_image(const dvg_scene_desc* desc, const dvg_render_options* opts, float* out_w) {
    Scene sc = decode(desc);
    std::vector<float> w = build_weight_image(sc, make_spec(opts));
    std::memcpy(out_w, w.data(), w.size() * sizeof(float));
    return 0;
}

extern "C" int oracle_sample_premultiplied(const dvg_scene_desc* desc, const dvg_render_options* opts, float px,
                                           float py, float* out4) {
    (void)opts;
    Scene sc = decode(desc);
    SceneBvh bvh = build_scene_bvh(sc);
    int x = to_i32(std::floor(px)), y = to_i32(std::floor(py));
    size_t pix = (x >= 0 && y >= 0 && x < (int)sc.w && y < (int)sc.h) ? (size_t)y * sc.w + x : 0;
    V4 c = eval_premultiplied(sc, bvh, mk(px, py), sample_background(sc, pix));
    out4[0] = c.x;
    out4[1] = c.y;
    out4[2] = c.z;
    out4[3] = c.w;
    return 0;
}

// Forward image with the crate's GPU semantics: rasterize_weights_f32, rasterize_splat_f32
// and resolve_splat_f32 (src/gpu/kernels/forward.rs:1505-1735, 294-334), with the early
// outs of Renderer::render (src/renderer/renderer.rs:40-66).
//
// oracle_render_window restricts the same computation to the pixels [x0,x1) x [y0,y1):
// a pixel's weight and colour sums receive only the samples of pixels within
// ceil(radius) of it, visited in increasing sample index as in the full render, so the
// window's pixels come out bit for bit as in the full image.  `threads` > 1 evaluates
// the per-sample colours on that many host threads; the weight and splat sums stay
// serial in sample order (same result for any thread count).
extern "C" int oracle_render_window(const dvg_scene_desc* desc, const dvg_render_options* opts, uint32_t x0,
                                    uint32_t y0, uint32_t x1, uint32_t y1, int threads, float* out) {
    Scene sc = decode(desc);
    if (sc.w == 0 || sc.h == 0) return 0;
    x1 = std::min<uint32_t>(x1, sc.w);
    y1 = std::min<uint32_t>(y1, sc.h);
    if (x0 >= x1 || y0 >= y1) return 0;
    const int width = (int)sc.w, height = (int)sc.h;
    const int ww = (int)(x1 - x0), wh = (int)(y1 - y0);
    const size_t wpix = (size_t)ww * wh;
    if (sc.groups.empty()) {
        for (int y = (int)y0; y < (int)y1; ++y)
            for (int x = (int)x0; x < (int)x1; ++x) {
                const size_t i = (size_t)y * width + x, o = (size_t)(y - (int)y0) * ww + (x - (int)x0);
                if (sc.has_bg_img)
                    for (int k = 0; k < 4; ++k) out[4 * o + k] = sc.bg_img[4 * i + k];
                else {
                    out[4 * o] = sc.bg.r;
                    out[4 * o + 1] = sc.bg.g;
                    out[4 * o + 2] = sc.bg.b;
                    out[4 * o + 3] = sc.bg.a;
                }
            }
        return 0;
    }
    SampleSpec sp = make_spec(opts);
    SceneBvh bvh = build_scene_bvh(sc);
    int ri = to_i32(std::ceil(sc.filter_radius));
    if (ri < 0) ri = 0;
    const uint64_t spp = (uint64_t)sp.sx_n * sp.sy_n;
    // pixels whose samples can reach the window
    const int ex0 = std::max(0, (int)x0 - ri), ey0 = std::max(0, (int)y0 - ri);
    const int ex1 = std::min(width, (int)x1 + ri), ey1 = std::min(height, (int)y1 + ri);
    const int ew = ex1 - ex0, eh = ey1 - ey0;
    const uint64_t esamples = (uint64_t)ew * eh * spp;
    auto sample_idx = [&](uint64_t k) {  // k-th sample of the extended window, in sample-index order
        const uint64_t s = k % spp, p = k / spp;
        const int x = ex0 + (int)(p % (uint64_t)ew), y = ey0 + (int)(p / (uint64_t)ew);
        return ((uint64_t)y * width + x) * spp + s;
    };
    std::vector<V4> colors(esamples);
    std::vector<V2> pts(esamples);
    parallel_for(0, esamples, threads, [&](int, uint64_t lo, uint64_t hi) {
        for (uint64_t k = lo; k < hi; ++k) {
            V2 pt;
            size_t pix;
            sample_position(sc, sp, sample_idx(k), &pt, &pix);
            pts[k] = pt;
            colors[k] = sp.prefilter ? eval_premultiplied_prefiltered(sc, bvh, pt, sample_background(sc, pix))
                                     : eval_premultiplied(sc, bvh, pt, sample_background(sc, pix));
        }
    });
    auto in_window = [&](int xx, int yy) { return xx >= (int)x0 && yy >= (int)y0 && xx < (int)x1 && yy < (int)y1; };
    std::vector<float> wimg(wpix, 0.0f);
    for (uint64_t k = 0; k < esamples; ++k) {
        const uint64_t p = k / spp;
        const int x = ex0 + (int)(p % (uint64_t)ew), y = ey0 + (int)(p / (uint64_t)ew);
        const V2 pt = pts[k];
        for (int dy = -ri; dy <= ri; ++dy)
            for (int dx = -ri; dx <= ri; ++dx) {
                int xx = x + dx, yy = y + dy;
                if (xx >= 0 && yy >= 0 && xx < width && yy < height && in_window(xx, yy)) {
                    float w = compute_filter_weight(sc.filter_type, sc.filter_radius, (float)xx + 0.5f - pt.x,
                                                    (float)yy + 0.5f - pt.y);
                    if (w > 0.0f) wimg[(size_t)(yy - (int)y0) * ww + (xx - (int)x0)] += w;
                }
            }
    }
    std::vector<float> acc(wpix * 4, 0.0f);
    for (uint64_t k = 0; k < esamples; ++k) {
        const uint64_t p = k / spp;
        const int x = ex0 + (int)(p % (uint64_t)ew), y = ey0 + (int)(p / (uint64_t)ew);
        const V2 pt = pts[k];
        const V4 c = colors[k];
        for (int dy = -ri; dy <= ri; ++dy)
            for (int dx = -ri; dx <= ri; ++dx) {
                int xx = x + dx, yy = y + dy;
                if (xx >= 0 && yy >= 0 && xx < width && yy < height && in_window(xx, yy)) {
                    size_t b = (size_t)(yy - (int)y0) * ww + (xx - (int)x0);
                    float ws = wimg[b];
                    if (ws > 0.0f) {
                        float w = compute_filter_weight(sc.filter_type, sc.filter_radius, (float)xx + 0.5f - pt.x,
                                                        (float)yy + 0.5f - pt.y);
                        if (w > 0.0f) {
                            float wn = w / ws;
                            acc[4 * b] += c.x * wn;
                            acc[4 * b + 1] += c.y * wn;
                            acc[4 * b + 2] += c.z * wn;
                            acc[4 * b + 3] += c.w * wn;
                        }
                    }
                }
            }
    }
    for (size_t i = 0; i < wpix; ++i) {
        float r = sc.bg.r, g = sc.bg.g, b = sc.bg.b, a = sc.bg.a;
        if (wimg[i] > 0.0f) {
            r = acc[4 * i];
            g = acc[4 * i + 1];
            b = acc[4 * i + 2];
            a = acc[4 * i + 3];
        }
        if (a > 1.0e-8f) {
            r = r / a;
            g = g / a;
            b = b / a;
        }
        out[4 * i] = r;
        out[4 * i + 1] = g;
        out[4 * i + 2] = b;
        out[4 * i + 3] = a;
    }
    return 0;
}

extern "C" int oracle_render(const dvg_scene_desc* desc, const dvg_render_options* opts, float* out) {
    return oracle_render_window(desc, opts, 0, 0, desc->width, desc->height, 1, out);
}

extern "C" int oracle_render_backward_ex(const dvg_scene_desc* desc, const dvg_render_options* opts,
                                         const dvg_backward_options* bopts, const float* d_render, dvg_grads* out,
                                         int passes, int threads, unsigned long long sample_begin,
                                         unsigned long long sample_end) {
    Scene sc = decode(desc);
    bool translation = bopts && bopts->compute_translation;
    bool include_bg_img = d_render != nullptr && sc.has_bg_img;
    Grads grads;
    grads.init(sc, desc, include_bg_img, translation);
    if (sc.w == 0 || sc.h == 0) {
        export_grads(grads, out, desc);
        return 0;
    }
    SampleSpec sp = make_spec(opts);
    uint64_t total = (uint64_t)sc.w * sc.h * sp.sx_n * sp.sy_n;
    SceneBvh bvh = build_scene_bvh(sc);
    if (d_render) {
        std::vector<float> wimg = build_weight_image(sc, sp);
        int nthreads = threads > 1 ? threads : 1;
        std::vector<Grads> tg(nthreads);
        for (auto& g : tg) g.init(sc, desc, include_bg_img, translation);
        if (passes & 1) {
            uint64_t b = sample_begin, e = sample_end ? std::min<uint64_t>(sample_end, total) : total;
            parallel_for(b, e, nthreads, [&](int t, uint64_t lo, uint64_t hi) {
                for (uint64_t idx = lo; idx < hi; ++idx) interior_sample(sc, bvh, sp, idx, d_render, wimg, tg[t], translation);
            });
        }
        if ((passes & 2) && !sp.prefilter) {
            BoundaryTables bt = build_boundary_tables(sc);
            if (bt.ok) {
                uint64_t nb = bopts && bopts->boundary_samples ? bopts->boundary_samples : total;
                uint32_t rng = bopts ? bopts->rng : 0;
                uint32_t seed = (bopts && !bopts->boundary_seed_from_options) ? bopts->boundary_seed : opts->seed;
                uint64_t b = sample_begin, e = sample_end ? std::min<uint64_t>(sample_end, nb) : nb;
                const float scale = (float)((double)nb / (double)total);
                parallel_for(b, e, nthreads, [&](int t, uint64_t lo, uint64_t hi) {
                    for (uint64_t idx = lo; idx < hi; ++idx)
                        boundary_sample(sc, bvh, bt, idx, rng, seed, d_render, wimg, tg[t], translation, scale);
                });
            }
        }
        for (auto& g : tg) grads.add(g);
    }
    finalize_background_gradients(sc, grads);
    export_grads(grads, out, desc);
    return 0;
}

// Deterministic expectation of the boundary pass: the crate draws N = W*H*spp samples,
// each a shape-cdf entry s (probability pmf_s) and a parameter t ~ U[0,1), so its boundary
// gradients average over seeds to N * sum_s pmf_s * integral_0^1 edge(s, t) dt.  The
// integral is taken by the midpoint rule, t_j = (j + 1/2) / m, every term through the same
// boundary_eval as a drawn sample.  offset as in boundary_eval (1e-4 for the crate).
extern "C" int oracle_boundary_integral(const dvg_scene_desc* desc, const dvg_render_options* opts,
                                        const float* d_render, uint32_t m, float offset, int threads, dvg_grads* out) {
    Scene sc = decode(desc);
    Grads grads;
    grads.init(sc, desc, false, false);
    SampleSpec sp = make_spec(opts);
    if (sc.w == 0 || sc.h == 0 || m == 0 || !d_render || sp.prefilter) {
        export_grads(grads, out, desc);
        return 0;
    }
    SceneBvh bvh = build_scene_bvh(sc);
    std::vector<float> wimg = build_weight_image(sc, sp);
    BoundaryTables bt = build_boundary_tables(sc);
    if (bt.ok) {
        const double n_samples = (double)sc.w * sc.h * sp.sx_n * sp.sy_n;
        const uint64_t entries = bt.cdf.shape_ids.size();
        int nthreads = threads > 1 ? threads : 1;
        std::vector<Grads> tg(nthreads);
        for (auto& g : tg) g.init(sc, desc, false, false);
        parallel_for(0, entries * m, nthreads, [&](int th, uint64_t lo, uint64_t hi) {
            for (uint64_t k = lo; k < hi; ++k) {
                const size_t e = (size_t)(k / m);
                const float pmf = e < bt.cdf.pmf.size() ? bt.cdf.pmf[e] : 0.0f;
                if (pmf <= 0.0f) continue;
                const float t = (float)(((double)(k % m) + 0.5) / m);
                boundary_eval(sc, bvh, bt, e, t, d_render, wimg, tg[th], false, 1.0f,
                              (float)(n_samples * pmf / m), offset);
            }
        });
        for (auto& g : tg) grads.add(g);
    }
    export_grads(grads, out, desc);
    return 0;
}

// ---------------------------------------------------------------- signed distance field
// Closest boundary over all groups, last group first (gpu/kernels/sdf.rs:8-115 for the
// forward, backward/sampling.rs:14-68 for the backward; same search, strict `<`
// between groups).  `init` is the starting bound: 1e20 in the GPU forward kernel,
// infinity in the CPU backward.
static bool sdf_closest(const Scene& sc, const SceneBvh& bvh, V2 pt, float init, ClosestPoint* best, size_t* group) {
    float best_dist = init;
    bool found = false;
    for (size_t gi = sc.groups.size(); gi-- > 0;) {
        ClosestPoint hit;
        if (compute_distance_bvh(sc, bvh, gi, pt, best_dist, &hit) && hit.distance < best_dist) {
            best_dist = hit.distance;
            *best = hit;
            *group = gi;
            found = true;
        }
    }
    return found;
}
static float sdf_signed(const Scene& sc, const SceneBvh& bvh, V2 pt) {  // compute_signed_distance
    ClosestPoint best;
    size_t g = 0;
    if (!sdf_closest(sc, bvh, pt, 1.0e20f, &best, &g)) return 0.0f;
    const bool inside = sc.groups[g].fill >= 0 && is_inside_bvh(sc, bvh, g, pt);
    return inside ? -best.distance : best.distance;
}
// sample_distance (backward/sampling.rs:14-68): every sample passes the pixel's full
// d_dist (the crate does not divide it by the sample count).
static void sample_distance(const Scene& sc, const SceneBvh& bvh, V2 pt, float d_dist, Grads& g, long translation_index) {
    ClosestPoint best;
    size_t gi = 0;
    if (!sdf_closest(sc, bvh, pt, INF_F, &best, &gi)) return;
    const bool inside = sc.groups[gi].fill >= 0 && is_inside_bvh(sc, bvh, gi, pt);
    const float d_abs = inside ? -d_dist : d_dist;
    PathInfo pinfo = path_info_from_closest(sc, best.shape_index, best.path);
    V2 d_pt = d_compute_distance(sc.groups[gi], gi, sc.shapes[best.shape_index], best.shape_index, pt, best.point, pinfo,
                                 d_abs, g);
    accumulate_translation(g, translation_index, d_pt * -1.0f);
}

// Renderer::render_sdf (renderer.rs:586-716, gpu/kernels/sdf.rs:118-200): per pixel the
// mean signed distance of its samples, at the GPU kernel's sample positions
// (x + (sx + r) * (1/sx_n)), jitter off when prefiltering.
extern "C" int oracle_render_sdf(const dvg_scene_desc* desc, const dvg_render_options* opts, float* out) {
    Scene sc = decode(desc);
    const size_t npix = (size_t)sc.w * sc.h;
    for (size_t i = 0; i < npix; ++i) out[i] = 0.0f;
    if (npix == 0 || sc.groups.empty()) return 0;
    SceneBvh bvh = build_scene_bvh(sc);
    const uint32_t sxn = opts->samples_x ? opts->samples_x : 1, syn = opts->samples_y ? opts->samples_y : 1;
    const bool jitter = !opts->use_prefiltering && opts->jitter;
    const float inv_sx = 1.0f / (float)sxn, inv_sy = 1.0f / (float)syn;
    const float inv_n = 1.0f / (float)(sxn * syn);
    for (uint32_t y = 0; y < sc.h; ++y)
        for (uint32_t x = 0; x < sc.w; ++x) {
            float acc = 0.0f;
            for (uint32_t sy = 0; sy < syn; ++sy)
                for (uint32_t sx = 0; sx < sxn; ++sx) {
                    float rx = 0.5f, ry = 0.5f;
                    if (jitter) {
                        uint64_t idx = (((uint64_t)y * sc.w + x) * syn + sy) * sxn + sx;
                        Pcg32 rng(idx, (uint64_t)opts->seed);
                        rx = rng.next_f32();
                        ry = rng.next_f32();
                    }
                    V2 pt = mk((float)x + ((float)sx + rx) * inv_sx, (float)y + ((float)sy + ry) * inv_sy);
                    acc += sdf_signed(sc, bvh, pt);
                }
            out[(size_t)y * sc.w + x] = acc * inv_n;
        }
    return 0;
}

// Renderer::eval_positions (renderer.rs:719-848, gpu/kernels/sdf.rs:203-262).
extern "C" int oracle_eval_positions(const dvg_scene_desc* desc, const float* positions, uint64_t n, float* out) {
    Scene sc = decode(desc);
    if (sc.groups.empty()) {
        for (uint64_t i = 0; i < n; ++i) out[i] = 0.0f;
        return 0;
    }
    SceneBvh bvh = build_scene_bvh(sc);
    for (uint64_t i = 0; i < n; ++i) out[i] = sdf_signed(sc, bvh, mk(positions[2 * i], positions[2 * i + 1]));
    return 0;
}

// The d_sdf_image part of render_backward (backward/render.rs:171-188): every sample of
// pixel p (CPU sample positions) passes d_sdf[p] to sample_distance.
extern "C" int oracle_sdf_backward(const dvg_scene_desc* desc, const dvg_render_options* opts,
                                   const dvg_backward_options* bopts, const float* d_sdf, dvg_grads* out) {
    Scene sc = decode(desc);
    bool translation = bopts && bopts->compute_translation;
    Grads grads;
    grads.init(sc, desc, false, translation);
    if (sc.w && sc.h && d_sdf) {
        SampleSpec sp = make_spec(opts);
        SceneBvh bvh = build_scene_bvh(sc);
        uint64_t total = (uint64_t)sc.w * sc.h * sp.sx_n * sp.sy_n;
        for (uint64_t idx = 0; idx < total; ++idx) {
            V2 pt;
            size_t pixel;
            sample_position(sc, sp, idx, &pt, &pixel);
            sample_distance(sc, bvh, pt, d_sdf[pixel], grads, translation ? (long)pixel : -1);
        }
    }
    finalize_background_gradients(sc, grads);
    export_grads(grads, out, desc);
    return 0;
}

// render_backward_positions (backward/render.rs:213-265).
extern "C" int oracle_positions_backward(const dvg_scene_desc* desc, const dvg_backward_options* bopts,
                                         const float* positions, uint64_t n, const float* d_values, dvg_grads* out) {
    Scene sc = decode(desc);
    bool translation = bopts && bopts->compute_translation;
    Grads grads;
    grads.init(sc, desc, false, translation);
    if (n && d_values) {
        SceneBvh bvh = build_scene_bvh(sc);
        for (uint64_t i = 0; i < n; ++i) {
            const float d = d_values[i];
            if (d == 0.0f) continue;
            V2 pt = mk(positions[2 * i], positions[2 * i + 1]);
            long ti = -1;
            if (translation) {  // translation_index_for_point (render.rs:267-281)
                int32_t x = to_i32(pt.x), y = to_i32(pt.y);
                if (x >= 0 && y >= 0 && x < (int32_t)sc.w && y < (int32_t)sc.h) ti = (long)y * (long)sc.w + x;
            }
            sample_distance(sc, bvh, pt, d, grads, ti);
        }
    }
    export_grads(grads, out, desc);
    return 0;
}

// ---------------------------------------------------------------- linear BVH (CPU twin)
// The same steps as the library's GPU build (Karras 2012): 16-bit-per-axis Morton
// codes of the box centres normalised to the centres' bounds (f32, no contraction),
// keys code << 32 | index sorted ascending, per-node range / split from common prefix
// lengths, bounds as exact unions.  Used to check the GPU tree bit for bit.
static uint32_t lb_spread16(uint32_t v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
static uint32_t lb_quantise(float c, float lo, float ext) {
    float u = ext > 0.0f ? (c - lo) / ext : 0.0f;
    u = std::fmin(std::fmax(u, 0.0f), 1.0f);
    const float s = u * 65536.0f;
    return s >= 65535.0f ? 65535u : (uint32_t)s;
}
static int lb_prefix(const std::vector<uint64_t>& k, int i, int j) {
    if (j < 0 || j >= (int)k.size()) return -1;
    return __builtin_clzll(k[i] ^ k[j]);
}
extern "C" int oracle_lbvh_build(const float* boxes, uint32_t count, uint64_t* keys_out, int32_t* children_out,
                                 float* bounds_out) {
    const int n = (int)count;
    if (n == 0) return 0;
    float x0 = INF_F, y0 = INF_F, x1 = -INF_F, y1 = -INF_F;
    for (int i = 0; i < n; ++i) {
        const float* b = boxes + 4 * i;
        const float cx = (b[0] + b[2]) * 0.5f, cy = (b[1] + b[3]) * 0.5f;
        x0 = std::fmin(x0, cx);
        y0 = std::fmin(y0, cy);
        x1 = std::fmax(x1, cx);
        y1 = std::fmax(y1, cy);
    }
    std::vector<uint64_t> keys(n);
    for (int i = 0; i < n; ++i) {
        const float* b = boxes + 4 * i;
        const float cx = (b[0] + b[2]) * 0.5f, cy = (b[1] + b[3]) * 0.5f;
        const uint32_t code = lb_spread16(lb_quantise(cx, x0, x1 - x0)) | (lb_spread16(lb_quantise(cy, y0, y1 - y0)) << 1);
        keys[i] = ((uint64_t)code << 32) | (uint32_t)i;
    }
    std::sort(keys.begin(), keys.end());
    std::vector<int> left(std::max(n - 1, 0)), right(std::max(n - 1, 0));
    for (int i = 0; i < n - 1; ++i) {
        const int d = lb_prefix(keys, i, i + 1) - lb_prefix(keys, i, i - 1) >= 0 ? 1 : -1;
        const int dmin = lb_prefix(keys, i, i - d);
        int lmax = 2;
        while (lb_prefix(keys, i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (lb_prefix(keys, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = lb_prefix(keys, i, j);
        int s = 0;
        for (int div = 2;; div *= 2) {
            const int t = (l + div - 1) / div;
            if (lb_prefix(keys, i, i + (s + t) * d) > dnode) s += t;
            if (t <= 1) break;
        }
        const int gamma = i + s * d + (d < 0 ? -1 : 0);
        left[i] = std::min(i, j) == gamma ? (n - 1) + gamma : gamma;
        right[i] = std::max(i, j) == gamma + 1 ? (n - 1) + gamma + 1 : gamma + 1;
    }
    std::vector<float> bounds(4 * (size_t)(2 * n - 1), 0.0f);
    for (int k = 0; k < n; ++k) {
        const float* b = boxes + 4 * (keys[k] & 0xffffffffu);
        for (int c = 0; c < 4; ++c) bounds[4 * (size_t)(n - 1 + k) + c] = b[c];
    }
    std::vector<int> stack, post;
    if (n > 1) stack.push_back(0);
    while (!stack.empty()) {  // post-order so children come before parents
        const int v = stack.back();
        stack.pop_back();
        post.push_back(v);
        if (left[v] < n - 1) stack.push_back(left[v]);
        if (right[v] < n - 1) stack.push_back(right[v]);
    }
    for (size_t q = post.size(); q-- > 0;) {
        const int v = post[q];
        const float* a = &bounds[4 * (size_t)left[v]];
        const float* b = &bounds[4 * (size_t)right[v]];
        float* o = &bounds[4 * (size_t)v];
        o[0] = std::fmin(a[0], b[0]);
        o[1] = std::fmin(a[1], b[1]);
        o[2] = std::fmax(a[2], b[2]);
        o[3] = std::fmax(a[3], b[3]);
    }
    if (keys_out) std::memcpy(keys_out, keys.data(), 8 * (size_t)n);
    if (children_out)
        for (int i = 0; i < n - 1; ++i) {
            children_out[2 * i] = left[i];
            children_out[2 * i + 1] = right[i];
        }
    if (bounds_out) std::memcpy(bounds_out, bounds.data(), bounds.size() * sizeof(float));
    return 0;
}

// The image the crate's render_backward differentiates: per pixel, the filter-
// weighted average of the CPU sample colours (un-premultiplied per sample, as
// backward/sampling.rs:76-224 returns them), with the weights gather_d_color
// uses (backward/filters.rs:70-103).  It equals the forward image wherever every
// sample of a pixel has alpha 1; pixels with no weight are 0.
extern "C" int oracle_render_differentiated(const dvg_scene_desc* desc, const dvg_render_options* opts, float* out) {
    Scene sc = decode(desc);
    if (sc.w == 0 || sc.h == 0) return 0;
    size_t npix = (size_t)sc.w * sc.h;
    std::fill(out, out + 4 * npix, 0.0f);
    SampleSpec sp = make_spec(opts);
    SceneBvh bvh = build_scene_bvh(sc);
    std::vector<float> wimg = build_weight_image(sc, sp);
    uint64_t total = (uint64_t)npix * sp.sx_n * sp.sy_n;
    int width = (int)sc.w, height = (int)sc.h;
    int ri = to_i32(std::ceil(sc.filter_radius));
    for (uint64_t idx = 0; idx < total; ++idx) {
        V2 pt;
        size_t pixel_index;
        sample_position(sc, sp, idx, &pt, &pixel_index);
        V2 npt = mk(pt.x / (float)sc.w, pt.y / (float)sc.h);
        V4 bg = sample_background(sc, pixel_index);
        V4 c = sp.prefilter ? sample_color_prefiltered(sc, bvh, npt, &bg, nullptr, nullptr, -1, pixel_index)
                            : sample_color(sc, bvh, npt, &bg, nullptr, nullptr, nullptr, -1, pixel_index);
        int x = to_i32(std::floor(pt.x)), y = to_i32(std::floor(pt.y));
        for (int dy = -ri; dy <= ri; ++dy)
            for (int dx = -ri; dx <= ri; ++dx) {
                int xx = x + dx, yy = y + dy;
                if (xx < 0 || yy < 0 || xx >= width || yy >= height) continue;
                float ws = wimg[(size_t)yy * width + xx];
                if (!(ws > 0.0f)) continue;
                float w = compute_filter_weight(sc.filter_type, sc.filter_radius, (float)xx + 0.5f - pt.x,
                                                (float)yy + 0.5f - pt.y);
                float* o = out + 4 * ((size_t)yy * width + xx);
                o[0] += (w / ws) * c.x;
                o[1] += (w / ws) * c.y;
                o[2] += (w / ws) * c.z;
                o[3] += (w / ws) * c.w;
            }
    }
    return 0;
}

extern "C" int oracle_render_backward(const dvg_scene_desc* desc, const dvg_render_options* opts,
                                      const dvg_backward_options* bopts, const float* d_render, dvg_grads* out) {
    return oracle_render_backward_ex(desc, opts, bopts, d_render, out, 3, 1, 0, 0);
}

extern "C" int oracle_compute_distance(const dvg_scene_desc* desc, uint32_t group, float px, float py,
                                       float max_radius, int use_bvh, float* out4) {
    Scene sc = decode(desc);
    ClosestPoint cp;
    bool ok;
    if (use_bvh) {
        SceneBvh bvh = build_scene_bvh(sc);
        ok = compute_distance_bvh(sc, bvh, group, mk(px, py), max_radius, &cp);
    } else {
        ok = compute_distance(sc, group, mk(px, py), max_radius, &cp);
    }
    if (!ok) return 0;
    out4[0] = (float)cp.shape_index;
    out4[1] = cp.point.x;
    out4[2] = cp.point.y;
    out4[3] = cp.distance;
    return 1;
}

extern "C" int oracle_within_distance(const dvg_scene_desc* desc, uint32_t group, float px, float py, int use_bvh) {
    Scene sc = decode(desc);
    if (use_bvh) {
        SceneBvh bvh = build_scene_bvh(sc);
        return within_distance_bvh(sc, bvh, group, mk(px, py)) ? 1 : 0;
    }
    return within_distance(sc, group, mk(px, py)) ? 1 : 0;
}

extern "C" int oracle_is_inside(const dvg_scene_desc* desc, uint32_t group, float px, float py, int use_bvh) {
    Scene sc = decode(desc);
    if (use_bvh) {
        SceneBvh bvh = build_scene_bvh(sc);
        return is_inside_bvh(sc, bvh, group, mk(px, py)) ? 1 : 0;
    }
    return is_inside(sc, group, mk(px, py)) ? 1 : 0;
}

// Path::flatten (geometry.rs:206-308) — recursive subdivision of quadratic / cubic segments.
namespace orc {
static float distance_point_line(V2 p, V2 a, V2 b) {  // geometry.rs:493-503
    V2 ab = b - a, ap = p - a;
    float area = std::fabs(cross(ab, ap));
    float len = length(ab);
    return len == 0.0f ? length(ap) : area / len;
}
static void flatten_quad(V2 p0, V2 p1, V2 p2, float tol, uint32_t depth, std::vector<V2>& out) {
    if (depth >= 16 || distance_point_line(p1, p0, p2) <= tol) {
        out.push_back(p0);
        out.push_back(p2);
        return;
    }
    V2 p01 = lerp(p0, p1, 0.5f), p12 = lerp(p1, p2, 0.5f), p012 = lerp(p01, p12, 0.5f);
    flatten_quad(p0, p01, p012, tol, depth + 1, out);
    flatten_quad(p012, p12, p2, tol, depth + 1, out);
}
static void flatten_cubic(V2 p0, V2 p1, V2 p2, V2 p3, float tol, uint32_t depth, std::vector<V2>& out) {
    float d = std::fmax(distance_point_line(p1, p0, p3), distance_point_line(p2, p0, p3));
    if (depth >= 16 || d <= tol) {
        out.push_back(p0);
        out.push_back(p3);
        return;
    }
    V2 p01 = lerp(p0, p1, 0.5f), p12 = lerp(p1, p2, 0.5f), p23 = lerp(p2, p3, 0.5f);
    V2 p012 = lerp(p01, p12, 0.5f), p123 = lerp(p12, p23, 0.5f), p0123 = lerp(p012, p123, 0.5f);
    flatten_cubic(p0, p01, p012, p0123, tol, depth + 1, out);
    flatten_cubic(p0123, p123, p23, p3, tol, depth + 1, out);
}
}  // namespace orc

extern "C" int oracle_flatten(const dvg_scene_desc* desc, uint32_t shape, float tolerance, float* out, int cap) {
    Scene sc = decode(desc);
    if (shape >= sc.shapes.size() || sc.shapes[shape].kind != DVG_SHAPE_PATH) return 0;
    const PathG& p = sc.shapes[shape].path;
    std::vector<V2> segs;
    if (p.ncp.empty() || p.pts.empty()) return 0;
    size_t point_id = 0;
    for (uint8_t nc : p.ncp) {
        V2 q[4];
        if (nc == 0) {
            if (!path_point(p, point_id, &q[0]) || !path_point(p, point_id + 1, &q[1])) break;
            segs.push_back(q[0]);
            segs.push_back(q[1]);
            point_id += 1;
        } else if (nc == 1) {
            if (!path_point(p, point_id, &q[0]) || !path_point(p, point_id + 1, &q[1]) ||
                !path_point(p, point_id + 2, &q[2]))
                break;
            flatten_quad(q[0], q[1], q[2], tolerance, 0, segs);
            point_id += 2;
        } else if (nc == 2) {
            if (!path_point(p, point_id, &q[0]) || !path_point(p, point_id + 1, &q[1]) ||
                !path_point(p, point_id + 2, &q[2]) || !path_point(p, point_id + 3, &q[3]))
                break;
            flatten_cubic(q[0], q[1], q[2], q[3], tolerance, 0, segs);
            point_id += 3;
        } else {
            break;
        }
    }
    int n = (int)(segs.size() / 2);
    for (int i = 0; i < n && i < cap; ++i) {
        out[4 * i] = segs[2 * i].x;
        out[4 * i + 1] = segs[2 * i].y;
        out[4 * i + 2] = segs[2 * i + 1].x;
        out[4 * i + 3] = segs[2 * i + 1].y;
    }
    return n;
}

extern "C" void oracle_pcg32_floats(unsigned long long idx, unsigned long long seed, int n, float* out) {
    Pcg32 rng(idx, seed);
    for (int i = 0; i < n; ++i) out[i] = rng.next_f32();
}

extern "C" void oracle_philox_floats(unsigned long long idx, unsigned int seed, float* out2) {
    boundary_rng(DVG_RNG_PHILOX, idx, seed, &out2[0], &out2[1]);
}

extern "C" int oracle_path_bvh(const dvg_scene_desc* desc, uint32_t shape, float* nodes, int node_cap, int* indices,
                               int index_cap, int* num_indices) {
    Scene sc = decode(desc);
    if (shape >= sc.shapes.size()) return 0;
    PathBvh pb;
    if (!build_path_bvh(sc.shapes[shape], &pb)) return 0;
    int n = (int)pb.nodes.size();
    for (int i = 0; i < n && i < node_cap; ++i) {
        const BvhNode& nd = pb.nodes[i];
        float* o = nodes + 8 * i;
        o[0] = nd.bounds.min.x;
        o[1] = nd.bounds.min.y;
        o[2] = nd.bounds.max.x;
        o[3] = nd.bounds.max.y;
        o[4] = nd.left == BVH_NONE ? -1.0f : (float)nd.left;
        o[5] = nd.right == BVH_NONE ? -1.0f : (float)nd.right;
        o[6] = (float)nd.start;
        o[7] = (float)nd.count;
    }
    *num_indices = (int)pb.indices.size();
    for (int i = 0; i < (int)pb.indices.size() && i < index_cap; ++i) indices[i] = (int)pb.indices[i];
    return n;
}

// Work of one forward pass, for the compute roofline: every test the crate's BVH
// queries reach when evaluated without early exits (is_inside_bvh, api.rs:259-309,
// within_distance_bvh, api.rs:79-135), for every pixel sample of the options.  A shape
// is reached when its group-space bounds (padded by the stroke radius, shape.rs:9-14)
// contain the sample; a path segment when its padded bounds pass the +x ray test (fill,
// winding.rs:117-126) or contain the sample (stroke, closest.rs:20-98).  Kinds: 0-2
// fill line / quadratic / cubic segment, 3-5 stroke line / quadratic / cubic segment,
// 6-8 fill circle / ellipse / rect, 9-11 stroke circle / ellipse / rect.  counts[k] =
// tests of kind k; flops[k] = the floating-point operations the crate's arithmetic
// executes for them (the winding solve, or the closest point plus radius), counted by
// OPS().  Needs the counting build (-DORACLE_COUNT_OPS); returns -1 otherwise.
extern "C" int oracle_count_work(const dvg_scene_desc* desc, const dvg_render_options* opts, int threads,
                                 unsigned long long* counts, unsigned long long* flops) {
    for (int i = 0; i < 12; ++i) counts[i] = flops[i] = 0;
#ifndef ORACLE_COUNT_OPS
    (void)desc;
    (void)opts;
    (void)threads;
    return -1;
#else
    Scene sc = decode(desc);
    SampleSpec sp = make_spec(opts);
    SceneBvh bvh = build_scene_bvh(sc);
    const uint64_t total = (uint64_t)sc.w * sc.h * sp.sx_n * sp.sy_n;
    const int nt = threads > 1 ? threads : 1;
    std::vector<std::vector<uint64_t>> tc(nt, std::vector<uint64_t>(24, 0));
    parallel_for(0, total, nt, [&](int t, uint64_t lo, uint64_t hi) {
        uint64_t* c = tc[t].data();
        uint64_t* f = c + 12;
        for (uint64_t idx = lo; idx < hi; ++idx) {
            V2 pt;
            size_t pix;
            sample_position(sc, sp, idx, &pt, &pix);
            for (size_t gi = 0; gi < sc.groups.size(); ++gi) {
                const Group& g = sc.groups[gi];
                if (g.fill < 0 && g.stroke < 0) continue;
                const V2 lp = xform_pt(g.c2s, pt);
                for (const BvhShape& bs : bvh.groups[gi].shapes) {
                    if (!bs.bounds.contains(lp)) continue;
                    const Shape& s = sc.shapes[bs.shape_index];
                    const bool stroke = g.stroke >= 0 && s.stroke_width > 0.0f;
                    if (s.kind == DVG_SHAPE_PATH) {
                        if (!bs.has_path_bvh) continue;
                        const V2 spt = xform_inv_dist(s.transform, lp);
                        for (const SegData& seg : bs.path_bvh.segments) {
                            const Bounds& b = seg.bounds;
                            if (g.fill >= 0 && !(spt.y < b.min.y || spt.y > b.max.y || spt.x > b.max.x)) {
                                g_ops = 0;
                                winding_number_segment(seg.kind, seg.p0, seg.p1, seg.p2, seg.p3, spt);
                                c[seg.kind] += 1;
                                f[seg.kind] += g_ops;
                            }
                            if (stroke && b.contains(spt)) {
                                g_ops = 0;
                                const CP cp = seg_closest(seg, spt, bs.path_bvh.approx);
                                seg_radius(seg, cp.t);
                                c[3 + seg.kind] += 1;
                                f[3 + seg.kind] += g_ops;
                            }
                        }
                        continue;
                    }
                    const int k = s.kind == DVG_SHAPE_CIRCLE ? 0 : s.kind == DVG_SHAPE_ELLIPSE ? 1 : 2;
                    if (g.fill >= 0) {
                        g_ops = 0;
                        winding_number_shape(s, nullptr, xform_inv_dist(s.transform, lp));
                        c[6 + k] += 1;
                        f[6 + k] += g_ops;
                    }
                    if (stroke) {
                        g_ops = 0;
                        within_distance_shape(s, lp, s.stroke_width);
                        c[9 + k] += 1;
                        f[9 + k] += g_ops;
                    }
                }
            }
        }
    });
    for (const auto& v : tc)
        for (int i = 0; i < 12; ++i) {
            counts[i] += v[i];
            flops[i] += v[12 + i];
        }
    return 0;
#endif
}

// Bounded-sample forward + backward for CPU timing: `count` samples spread evenly
// over the W*H*spp sample sequence (idx = k*stride), each doing the forward
// per-sample evaluation (premultiplied colour and filtered splat) and the interior
// adjoint, plus count*nb/total boundary samples spread the same way over the
// nb-sample boundary pass.  Runs on `threads` host threads with per-thread gradient
// buffers, as a parallel port of the crate's serial loops
// (src/backward/render.rs:95-205).  Writes the per-call set-up time (BVH, weight
// image, CDF tables) and the sample-loop time in seconds to times[0..1].
extern "C" unsigned long long oracle_fwd_bwd_sample(const dvg_scene_desc* desc, const dvg_render_options* opts,
                                                    const dvg_backward_options* bopts, const float* d_render,
                                                    unsigned long long count, int threads, double* times) {
    auto now = []() { return std::chrono::steady_clock::now(); };
    auto t0 = now();
    Scene sc = decode(desc);
    if (sc.w == 0 || sc.h == 0 || sc.groups.empty()) return 0;
    SampleSpec sp = make_spec(opts);
    uint64_t total = (uint64_t)sc.w * sc.h * sp.sx_n * sp.sy_n;
    if (count > total) count = total;
    if (count == 0) return 0;
    uint64_t stride = total / count;
    SceneBvh bvh = build_scene_bvh(sc);
    std::vector<float> wimg = build_weight_image(sc, sp);
    BoundaryTables bt = build_boundary_tables(sc);
    int nthreads = threads > 1 ? threads : 1;
    std::vector<Grads> tg(nthreads);
    std::vector<std::vector<float>> acc(nthreads);
    for (int t = 0; t < nthreads; ++t) {
        tg[t].init(sc, desc, false, false);
        acc[t].assign((size_t)sc.w * sc.h * 4, 0.0f);
    }
    auto t1 = now();
    int ri = std::max(0, to_i32(std::ceil(sc.filter_radius)));
    int width = (int)sc.w, height = (int)sc.h;
    parallel_for(0, count, nthreads, [&](int t, uint64_t lo, uint64_t hi) {
        for (uint64_t k = lo; k < hi; ++k) {
            uint64_t idx = k * stride;
            V2 pt;
            size_t pix;
            sample_position(sc, sp, idx, &pt, &pix);
            V4 c = sp.prefilter ? eval_premultiplied_prefiltered(sc, bvh, pt, sample_background(sc, pix))
                                : eval_premultiplied(sc, bvh, pt, sample_background(sc, pix));
            int x = (int)(pix % sc.w), y = (int)(pix / sc.w);
            for (int dy = -ri; dy <= ri; ++dy)
                for (int dx = -ri; dx <= ri; ++dx) {
                    int xx = x + dx, yy = y + dy;
                    if (xx < 0 || yy < 0 || xx >= width || yy >= height) continue;
                    size_t b = (size_t)yy * width + xx;
                    float w = compute_filter_weight(sc.filter_type, sc.filter_radius, (float)xx + 0.5f - pt.x,
                                                    (float)yy + 0.5f - pt.y);
                    if (w > 0.0f && wimg[b] > 0.0f) {
                        float wn = w / wimg[b];
                        acc[t][4 * b] += c.x * wn;
                        acc[t][4 * b + 1] += c.y * wn;
                        acc[t][4 * b + 2] += c.z * wn;
                        acc[t][4 * b + 3] += c.w * wn;
                    }
                }
            interior_sample(sc, bvh, sp, idx, d_render, wimg, tg[t], false);
        }
    });
    if (bt.ok && !sp.prefilter) {
        uint64_t nb = bopts && bopts->boundary_samples ? bopts->boundary_samples : total;
        uint64_t bcount = count * nb / total;
        uint64_t bstride = bcount ? nb / bcount : 1;
        uint32_t rng = bopts ? bopts->rng : 0;
        uint32_t seed = (bopts && !bopts->boundary_seed_from_options) ? bopts->boundary_seed : opts->seed;
        const float scale = (float)((double)nb / (double)total);
        parallel_for(0, bcount, nthreads, [&](int t, uint64_t lo, uint64_t hi) {
            for (uint64_t k = lo; k < hi; ++k)
                boundary_sample(sc, bvh, bt, k * bstride, rng, seed, d_render, wimg, tg[t], false, scale);
        });
    }
    auto t2 = now();
    if (times) {
        times[0] = std::chrono::duration<double>(t1 - t0).count();
        times[1] = std::chrono::duration<double>(t2 - t1).count();
    }
    return count;
}
