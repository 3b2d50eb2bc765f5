// winding_stress.cpp — test infrastructure: the certified f32 cubic winding of the
// library (diffvg-rs_b200/csrc/certified_f32.cuh) against the oracle's restatement of
// the crate's f64 computation (winding_number_segment, winding.rs:170-192), on random
// and adversarial segments.  Built into oracle/_build/libwinding_stress.so by the
// Makefile; driven by tests/test_winding_f32.py.
#include "oracle.cpp"

#include "../diffvg-rs_b200/csrc/certified_f32.cuh"

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

// mode 0: control points uniform in [-64, 64]^2, query points near the curve at a random
//         t plus an offset of random sign and magnitude 10^U[-6, 1.3];
// mode 1: integer control points in [-16, 16] and integer or half-integer query points
//         (exact alignments with end points and extrema);
// mode 2: near-degenerate cubics: elevated quadratics and lines with perturbations of
//         10^U[-7, -1], cusps and tiny loops;
// mode 3: query rows exactly at the end-point y values and at the y extrema;
// mode 4: coordinates scaled to |x| up to 4096;
// mode 5: the tests a scene makes: query points uniform over the control points' box.
// perturb > 0: every initial root is moved by up to +-perturb before the refinement
// and the certificate (the largest error of the GPU's fast root formulas is ~5e-4).
// out[0] = cases, out[1] = certified, out[2] = certified and different from f64.
static int winding_perturbed(const V2* p, V2 q, float perturb, SplitMix& rng) {
    const float a = -p[0].y + 3.0f * p[1].y - 3.0f * p[2].y + p[3].y;
    const float b = 3.0f * p[0].y - 6.0f * p[1].y + 3.0f * p[2].y;
    const float c = -3.0f * p[0].y + 3.0f * p[1].y;
    const float d = p[0].y - q.y;
    const float mcoef = std::fmax(std::fmax(std::fabs(b), std::fabs(c)), std::fabs(d));
    if (!(std::fabs(a) >= 1.0e-3f) || !(std::fabs(a) * 16.0f >= mcoef)) return dvgb::WIND_UNSURE;
    float t[3];
    const int n = dvgb::cubic_roots_f32(b / a, c / a, d / a, t);
    if (n < 0) return dvgb::WIND_UNSURE;
    for (int i = 0; i < n; ++i) t[i] += rng.range(-perturb, perturb);
    return dvgb::winding_from_roots(a, b, c, d, t, n, p[0].x, p[1].x, p[2].x, p[3].x, q.x);
}
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
        // query point
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
        if (mode == 3) {
            const int pick = (int)(rng.next() % 3);
            if (pick == 0) q.y = p[0].y;
            if (pick == 1) q.y = p[3].y;
            if (pick == 2) {  // a y extremum, from y'(t) = 0 in f64
                double a = -p[0].y + 3.0 * p[1].y - 3.0 * p[2].y + p[3].y, b = 3.0 * p[0].y - 6.0 * p[1].y + 3.0 * p[2].y,
                       c = -3.0 * p[0].y + 3.0 * p[1].y;
                double r[2];
                if (solve_quadratic(3.0 * a, 2.0 * b, c, r)) {
                    double tt = r[rng.next() % 2];
                    q.y = (float)(((a * tt + b) * tt + c) * tt + p[0].y);
                }
            }
        }
        const int ref = winding_number_segment(2, p[0], p[1], p[2], p[3], q);
        const int fast = perturb > 0.0f
                             ? winding_perturbed(p, q, perturb, rng)
                             : dvgb::winding_cubic_f32(p[0].x, p[0].y, p[1].x, p[1].y, p[2].x, p[2].y, p[3].x, p[3].y,
                                                       q.x, q.y);
        out[0] += 1;
        if (fast != dvgb::WIND_UNSURE) {
            out[1] += 1;
            if (fast != ref) out[2] += 1;
        }
    }
}

// The certified f32 stroke test of a quadratic segment (within_quad_f32) against the
// oracle's closest_point_quadratic (curve.rs:26-78) and the radius test (closest.rs:66-79).
// mode 0: control points uniform in [-64, 64]^2, radius U[0.5, 8], query points at
//         distance r + 10^U[-6, 1] (random sign) from a random curve point's normal;
// mode 1: nearly straight quadratics (p1 on the chord plus 10^U[-7, 0]);
// mode 2: degenerate ones (p1 = p0, p1 = p2, p0 = p2);
// mode 3: coordinates scaled up to 4096;
// mode 4: the tests a scene makes: query points uniform over the radius-padded box.
// perturb > 0: initial roots moved by up to +-perturb, as for the winding.
// out[0] = cases, out[1] = certified, out[2] = certified and different from f64.
static int within_perturbed(const V2* p, float r, V2 q, float perturb, SplitMix& rng) {
    const float ax = p[0].x - 2.0f * p[1].x + p[2].x, ay = p[0].y - 2.0f * p[1].y + p[2].y;
    const float bx = -p[0].x + p[1].x, by = -p[0].y + p[1].y;
    const float cx = p[0].x - q.x, cy = p[0].y - q.y;
    const float A = ax * ax + ay * ay;
    const float B = 3.0f * (ax * bx + ay * by);
    const float C = 2.0f * (bx * bx + by * by) + (ax * cx + ay * cy);
    const float D = bx * cx + by * cy;
    const float mcoef = std::fmax(std::fmax(std::fabs(B), std::fabs(C)), std::fabs(D));
    if (!(A >= 1.0e-3f) || !(A * 16.0f >= mcoef)) return dvgb::WITHIN_UNSURE;
    float t[3];
    const int n = dvgb::cubic_roots_f32(B / A, C / A, D / A, t);
    if (n < 0) return dvgb::WITHIN_UNSURE;
    for (int i = 0; i < n; ++i) t[i] += rng.range(-perturb, perturb);
    return dvgb::within_quad_from_roots(t, n, p[0].x, p[0].y, p[1].x, p[1].y, p[2].x, p[2].y, r, q.x, q.y, A, B, C, D);
}
extern "C" void within_stress(int mode, uint64_t seed, uint64_t n, float perturb, unsigned long long* out) {
    SplitMix rng{seed * 0x9e3779b97f4a7c15ull + 77 + (uint64_t)mode};
    out[0] = out[1] = out[2] = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const float scale = mode == 3 ? rng.range(64.0f, 4096.0f) : 64.0f;
        V2 p[3];
        for (int k = 0; k < 3; ++k) p[k] = mk(rng.range(-1.0f, 1.0f) * scale, rng.range(-1.0f, 1.0f) * scale);
        const float r = rng.range(0.5f, 8.0f) * (scale / 64.0f);
        if (mode == 1)
            p[1] = lerp(p[0], p[2], (float)rng.uni()) +
                   mk(rng.range(-1, 1), rng.range(-1, 1)) * (float)std::pow(10.0, -7.0 + 7.0 * rng.uni());
        if (mode == 2) {
            const int k = (int)(rng.next() % 3);
            if (k == 0) p[1] = p[0];
            if (k == 1) p[1] = p[2];
            if (k == 2) p[2] = p[0];
        }
        V2 q;
        if (mode == 4) {
            V2 lo = vmin(vmin(p[0], p[1]), p[2]), hi = vmax(vmax(p[0], p[1]), p[2]);
            q = mk(rng.range(lo.x - r, hi.x + r), rng.range(lo.y - r, hi.y + r));
        } else {
            const float t = (float)rng.uni(), u = 1.0f - t;
            const V2 on = p[0] * (u * u) + p[1] * (2.0f * u * t) + p[2] * (t * t);
            V2 tg = (p[1] - p[0]) * (2.0f * u) + (p[2] - p[1]) * (2.0f * t);
            float tl = length(tg);
            V2 nrm = tl > 0.0f ? mk(-tg.y / tl, tg.x / tl) : mk(1.0f, 0.0f);
            const float off = r + (rng.next() % 2 ? 1.0f : -1.0f) * (float)std::pow(10.0, -6.0 + 7.0 * rng.uni());
            q = on + nrm * off;
        }
        const CP c = closest_point_quadratic(q, p[0], p[1], p[2], false);
        const float tt = 1.0f - c.t;
        const int ref = c.dist < tt * tt * r + 2.0f * tt * c.t * r + c.t * c.t * r ? 1 : 0;
        const int fast = perturb > 0.0f ? within_perturbed(p, r, q, perturb, rng)
                                        : dvgb::within_quad_f32(p[0].x, p[0].y, p[1].x, p[1].y, p[2].x, p[2].y, r, q.x,
                                                                q.y);
        out[0] += 1;
        if (fast != dvgb::WITHIN_UNSURE) {
            out[1] += 1;
            if (fast != ref) out[2] += 1;
        }
    }
}
