// winding_stress.cpp — test infrastructure: the library's Newton-certified cubic winding
// (diffvg-rs_b200/csrc/winding_newton.cuh) against the oracle's restatement of the
// crate's f64 computation (winding_number_segment, winding.rs:170-192), on random and
// adversarial segments.  Built into oracle/_build/libwinding_stress.so by the Makefile;
// driven by tests/test_winding_newton.py.
#include "oracle.cpp"

#include "../diffvg-rs_b200/csrc/winding_newton.cuh"

namespace {
struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    float range(float lo, float hi) { return (float)(lo + (hi - lo) * uni()); }
};
}  // namespace

// The library's call: the crate's coefficient expressions (f32, then widened), as in
// winding_segment_v (device.cuh).
static int newton_winding(const V2* p, V2 q, const float* perturb) {
    const double a = (double)(-p[0].y + 3.0f * p[1].y - 3.0f * p[2].y + p[3].y);
    const double b = (double)(3.0f * p[0].y - 6.0f * p[1].y + 3.0f * p[2].y);
    const double c = (double)(-3.0f * p[0].y + 3.0f * p[1].y);
    const double d = (double)(p[0].y - q.y);
    const double ax = (double)(-p[0].x + 3.0f * p[1].x - 3.0f * p[2].x + p[3].x);
    const double bx = (double)(3.0f * p[0].x - 6.0f * p[1].x + 3.0f * p[2].x);
    const double cx = (double)(-3.0f * p[0].x + 3.0f * p[1].x);
    const double dx = (double)(p[0].x - q.x);
    return dvgb::winding_cubic_newton(a, b, c, d, ax, bx, cx, dx, perturb);
}

// mode 0: control points uniform in [-64, 64]^2, query points near the curve at a random
//         t plus an offset of random sign and magnitude 10^U[-6, 1.3];
// mode 1: integer control points in [-16, 16] and integer or half-integer query points
//         (exact alignments with end points and extrema);
// mode 2: near-degenerate cubics: elevated quadratics and lines with perturbations of
//         10^U[-7, -1], cusps and tiny loops;
// mode 3: query rows exactly at the end-point y values and at the y extrema;
// mode 4: coordinates scaled to |x| up to 4096;
// mode 5: the tests a scene makes: query points uniform over the control points' box;
// mode 6: near double roots: query rows within 10^U[-12, -2] of a y extremum.
// perturb > 0: every f32 root estimate moves by U[-perturb, perturb] times the scale of
// its formula before the Newton step (the device's fast cosine, with an absolute error
// near 2^-21, and its f32 formulas differ from the host's).
// out[0] = cases, out[1] = decided by the Newton path, out[2] = decided and different
// from the crate's f64 computation.
extern "C" void winding_stress(int mode, uint64_t seed, uint64_t n, float perturb, unsigned long long* out) {
    SplitMix rng{seed * 0x2545f4914f6cdd1dull + (uint64_t)mode};
    out[0] = out[1] = out[2] = 0;
    for (uint64_t i = 0; i < n; ++i) {
        V2 p[4];
        float scale = mode == 4 ? rng.range(64.0f, 4096.0f) : 64.0f;
        for (int k = 0; k < 4; ++k) p[k] = mk(rng.range(-1.0f, 1.0f) * scale, rng.range(-1.0f, 1.0f) * scale);
        if (mode == 1)
            for (int k = 0; k < 4; ++k) p[k] = mk(std::floor(rng.range(-16.0f, 17.0f)), std::floor(rng.range(-16.0f, 17.0f)));
        if (mode == 2) {
            const int kind = (int)(rng.next() % 4);
            const float eps = (float)std::pow(10.0, -7.0 + 6.0 * rng.uni());
            if (kind == 0) {  // elevated quadratic: p1, p2 on the quadratic's thirds
                V2 q1 = mk(rng.range(-64, 64), rng.range(-64, 64));
                p[1] = p[0] + (q1 - p[0]) * (2.0f / 3.0f);
                p[2] = p[3] + (q1 - p[3]) * (2.0f / 3.0f);
            } else if (kind == 1) {  // a line as a cubic
                p[1] = lerp(p[0], p[3], 1.0f / 3.0f);
                p[2] = lerp(p[0], p[3], 2.0f / 3.0f);
            } else if (kind == 2) {  // cusp: p1 and p2 swapped across the chord
                p[1] = lerp(p[0], p[3], 0.7f);
                p[2] = lerp(p[0], p[3], 0.3f);
            } else {  // tiny loop
                p[1] = p[3] + mk(rng.range(-4, 4), rng.range(-4, 4));
                p[2] = p[0] + mk(rng.range(-4, 4), rng.range(-4, 4));
            }
            for (int k = 1; k < 3; ++k) p[k] = p[k] + mk(rng.range(-1, 1) * eps * 64.0f, rng.range(-1, 1) * eps * 64.0f);
        }
        V2 q;
        const float t = (float)rng.uni();
        const float u = 1.0f - t;
        const V2 on = p[0] * (u * u * u) + p[1] * (3.0f * u * u * t) + p[2] * (3.0f * u * t * t) + p[3] * (t * t * t);
        if (mode == 5) {
            V2 lo = vmin(vmin(p[0], p[1]), vmin(p[2], p[3])), hi = vmax(vmax(p[0], p[1]), vmax(p[2], p[3]));
            q = mk(rng.range(lo.x, hi.x), rng.range(lo.y, hi.y));
        } else if (mode == 1) {
            q = mk(std::floor(rng.range(-17.0f, 18.0f)) * (rng.next() % 2 ? 1.0f : 0.5f),
                   std::floor(rng.range(-17.0f, 18.0f)) * (rng.next() % 2 ? 1.0f : 0.5f));
        } else {
            const float mag = (float)std::pow(10.0, -6.0 + 7.3 * rng.uni()) * (scale / 64.0f);
            q = on + mk(rng.range(-1, 1) * mag, rng.range(-1, 1) * mag);
        }
        if (mode == 3 || mode == 6) {
            const int pick = mode == 6 ? 2 : (int)(rng.next() % 3);
            if (pick == 0) q.y = p[0].y;
            if (pick == 1) q.y = p[3].y;
            if (pick == 2) {  // a y extremum, from y'(t) = 0 in f64
                double a = -p[0].y + 3.0 * p[1].y - 3.0 * p[2].y + p[3].y, b = 3.0 * p[0].y - 6.0 * p[1].y + 3.0 * p[2].y,
                       c = -3.0 * p[0].y + 3.0 * p[1].y;
                double r[2];
                if (solve_quadratic(3.0 * a, 2.0 * b, c, r)) {
                    double tt = r[rng.next() % 2];
                    double ye = ((a * tt + b) * tt + c) * tt + p[0].y;
                    if (mode == 6) ye += (rng.next() % 2 ? 1.0 : -1.0) * std::pow(10.0, -12.0 + 10.0 * rng.uni()) *
                                         (1.0 + std::fabs(ye));
                    q.y = (float)ye;
                }
            }
        }
        const int ref = winding_number_segment(2, p[0], p[1], p[2], p[3], q);
        float pert[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k) pert[k] = rng.range(-perturb, perturb);
        const int fast = newton_winding(p, q, perturb > 0.0f ? pert : nullptr);
        out[0] += 1;
        if (fast != dvgb::WIND_UNSURE) {
            out[1] += 1;
            if (fast != ref) out[2] += 1;
        }
    }
}

// The quadratic closest point from the certified candidates (closest_quad_roots_newton),
// the rest as the crate's closest_point_quadratic (curve.rs:26-78); -1 in *ok: not certain.
static CP newton_closest_quad(V2 pt, V2 p0, V2 p1, V2 p2, const float* perturb, int* ok) {
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
    float ts[3];
    const int n = dvgb::closest_quad_roots_newton(a, b, c, d, ts, perturb);
    *ok = n >= 0;
    for (int i = 0; i < n; ++i) {
        const float t32 = ts[i];
        const float tt = 1.0f - t32;
        V2 cp = (p0 * (tt * tt)) + (p1 * (2.0f * tt * t32)) + (p2 * (t32 * t32));
        float dist = length(pt - cp);
        if (dist < best_dist) {
            best_dist = dist;
            best_pt = cp;
            best_t = t32;
        }
    }
    return CP{best_pt, best_t, best_dist};
}

// mode 0: control points uniform in [-64, 64]^2, query points near a random curve point
//         (offset 10^U[-6, 1.3] in a random direction);
// mode 1: integer control points and integer or half-integer query points;
// mode 2: nearly straight and degenerate quadratics (p1 on the chord + 10^U[-7, 0], p1 = p0,
//         p1 = p2), query points near the curve;
// mode 3: query points near the centre of curvature of a random curve point (where two
//         stationary points merge);
// mode 4: the tests a scene makes: query points uniform over the box padded by 8.
// out[0] = cases, out[1] = decided, out[2] = decided and not bit-identical to the crate's
// (point, t, distance).
extern "C" void closest_quad_stress(int mode, uint64_t seed, uint64_t n, float perturb, unsigned long long* out) {
    SplitMix rng{seed * 0x9e3779b97f4a7c15ull + 101 + (uint64_t)mode};
    out[0] = out[1] = out[2] = 0;
    for (uint64_t i = 0; i < n; ++i) {
        V2 p[3];
        for (int k = 0; k < 3; ++k) p[k] = mk(rng.range(-64.0f, 64.0f), rng.range(-64.0f, 64.0f));
        if (mode == 1)
            for (int k = 0; k < 3; ++k) p[k] = mk(std::floor(rng.range(-16.0f, 17.0f)), std::floor(rng.range(-16.0f, 17.0f)));
        if (mode == 2) {
            const int kind = (int)(rng.next() % 3);
            if (kind == 0) {
                const float eps = (float)std::pow(10.0, -7.0 + 7.0 * rng.uni());
                p[1] = lerp(p[0], p[2], (float)rng.uni()) + mk(rng.range(-1, 1) * eps * 64.0f, rng.range(-1, 1) * eps * 64.0f);
            } else if (kind == 1) {
                p[1] = p[0];
            } else {
                p[1] = p[2];
            }
        }
        const float t = (float)rng.uni(), u = 1.0f - t;
        const V2 on = p[0] * (u * u) + p[1] * (2.0f * u * t) + p[2] * (t * t);
        V2 q;
        if (mode == 1) {
            q = mk(std::floor(rng.range(-17.0f, 18.0f)) * (rng.next() % 2 ? 1.0f : 0.5f),
                   std::floor(rng.range(-17.0f, 18.0f)) * (rng.next() % 2 ? 1.0f : 0.5f));
        } else if (mode == 3) {
            // centre of curvature: on + n * R, R = |B'|^3 / |B' x B''|
            const V2 d1 = (p[1] - p[0]) * (2.0f * u) + (p[2] - p[1]) * (2.0f * t);
            const V2 d2 = (p[2] - p[1] * 2.0f + p[0]) * 2.0f;
            const float cr = d1.x * d2.y - d1.y * d2.x, l = length(d1);
            if (!(std::fabs(cr) > 1e-6f)) continue;
            const float R = l * l * l / cr;
            const V2 nrm = mk(-d1.y / l, d1.x / l);
            const float jit = (float)std::pow(10.0, -6.0 + 5.0 * rng.uni()) * (rng.next() % 2 ? 1.0f : -1.0f);
            q = on + nrm * (R * (1.0f + jit));
        } else if (mode == 4) {
            V2 lo = vmin(vmin(p[0], p[1]), p[2]) - mk(8, 8), hi = vmax(vmax(p[0], p[1]), p[2]) + mk(8, 8);
            q = mk(rng.range(lo.x, hi.x), rng.range(lo.y, hi.y));
        } else {
            const float mag = (float)std::pow(10.0, -6.0 + 7.3 * rng.uni());
            const float ang = (float)(6.283185307179586 * rng.uni());
            q = on + mk(std::cos(ang) * mag, std::sin(ang) * mag);
        }
        const CP ref = closest_point_quadratic(q, p[0], p[1], p[2], false);
        float pert[3];
        for (int k = 0; k < 3; ++k) pert[k] = rng.range(-perturb, perturb);
        int ok = 0;
        const CP got = newton_closest_quad(q, p[0], p[1], p[2], perturb > 0.0f ? pert : nullptr, &ok);
        out[0] += 1;
        if (ok) {
            out[1] += 1;
            if (std::memcmp(&got, &ref, sizeof(CP)) != 0) out[2] += 1;
        }
    }
}
