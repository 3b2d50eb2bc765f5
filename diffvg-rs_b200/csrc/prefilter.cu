// prefilter.cu — prefiltered (smoothstep-coverage) forward and interior adjoint.
//
// RenderOptions::use_prefiltering (the crate's default): coverage comes from
// the signed distance to the closest boundary (src/backward/sampling.rs:227-482)
// instead of point sampling, so the interior adjoint also reaches the geometry
// through d_compute_distance (src/backward/distance.rs:50-561).  The closest-point
// search walks the crate's BVHs with an explicit stack in the crate's order
// (closer child first, src/distance/api.rs:138-236, closest.rs:104-199): the
// order only matters for exact distance ties, which it resolves the same way.
// Built with -fmad=false like kernels.cu.  The quadratic closest point runs the crate's
// root formula here (DVG_EXACT_CLOSEST_QUAD): these kernels call it for every segment
// within the distance search, and its certified shortcut measured slower in them (mixed
// 512x512 scene, 4x4 spp: prefiltered interior 65.8 ms without it, 66.9 with it).
#ifndef DVG_EXACT_CLOSEST_QUAD
#define DVG_EXACT_CLOSEST_QUAD 1
#endif
#include <algorithm>

#include "device.cuh"
#include "kernels.cuh"
// Minimum resident CTAs per SM of the prefiltered forward and interior kernels, by
// measurement on B200 (mixed 512x512 scene, 4x4 spp): the forward at 4 (64 registers,
// spilling) 42.0 -> 36.4 ms against 2; the interior at 1 (168 registers, no spills)
// 64.7 -> 62.6 ms against the compiler's own choice of 128.
#ifndef DVG_MINB_PF_FWD
#define DVG_MINB_PF_FWD 4
#endif
#ifndef DVG_MINB_PF_INT
#define DVG_MINB_PF_INT 1
#endif
// The per-sample signed-distance kernels (render_sdf and its adjoints) at 4 CTAs per SM
// (64 registers): render_sdf 75.1 -> 64.4 ms and its backward 44.4 -> 41.3 ms on the
// mixed 512x512 scene against the compiler's own 118-124 registers.
#ifndef DVG_MINB_SDF
#define DVG_MINB_SDF 4
#endif
#define DVG_SDF_BOUNDS __launch_bounds__(256, DVG_MINB_SDF)

namespace dvgb {

constexpr int BVH_STACK = 64;
constexpr float INF_F = __builtin_huge_valf();

__device__ __forceinline__ float box_distance(float4 b, float2 p) {  // Bounds::distance (bvh.rs:109-113)
    float dx = fmaxf(fmaxf(b.x - p.x, 0.0f), p.x - b.z);
    float dy = fmaxf(fmaxf(b.y - p.y, 0.0f), p.y - b.w);
    return sqrtf(dx * dx + dy * dy);
}

struct ClosestD {
    int shape;
    float2 point;  // canvas space
    float dist;
    int seg;  // segment index within the path, -1 when the shape is not a path
    float t;
};

// closest_point_path_bvh (closest.rs:104-199); cp in shape space.
static __device__ bool closest_path_bvh(const DevScene& S, int path, float2 p, float2* cp, int* seg, float* tt,
                                 unsigned* status) {
    const int4 pi = __ldg(&S.p_info[2 * path]);
    if (pi.w == 0) return false;
    const bool approx = __ldg(&S.p_info[2 * path + 1].w) & PF_APPROX;
    float best = INF_F, bt = 0.0f;
    float2 bp = make_float2(0.0f, 0.0f);
    int bseg = 0;
    int stk[BVH_STACK];
    int sp = 0;
    stk[sp++] = pi.z;
    int guard = 0;
    while (sp > 0 && guard++ < (1 << 20)) {
        const int n = stk[--sp];
        const int4 m = __ldg(&S.pn_meta[n]);
        if (box_distance(__ldg(&S.pn_bounds[n]), p) > best) continue;
        if (m.z > 0) {
            for (int k = m.y; k < m.y + m.z; ++k) {
                const int sidx = __ldg(&S.pl_segs[k]);
                SegGeom sg;
                load_seg(S, sidx, sg);
                if (cubic_cannot_beat(sg, p, approx, best)) continue;
                CPRes c = seg_closest(sg, p, approx);
                if (c.dist < best) {
                    best = c.dist;
                    bp = make_float2(c.cx, c.cy);
                    bseg = __ldg(&S.seg_meta[sidx].y);
                    bt = c.t;
                }
            }
        } else {
            const int l = n + 1, r = m.w;
            const float ld = box_distance(__ldg(&S.pn_bounds[l]), p);
            const float rd = r >= 0 ? box_distance(__ldg(&S.pn_bounds[r]), p) : INF_F;
            if (sp + 2 > BVH_STACK) {
                atomicOr(status, ST_BVH_LIMIT);
                break;
            }
            if (ld < rd) {
                if (rd <= best) stk[sp++] = r;
                if (ld <= best) stk[sp++] = l;
            } else {
                if (ld <= best) stk[sp++] = l;
                if (rd <= best) stk[sp++] = r;
            }
        }
    }
    if (!isfinite(best)) return false;
    *cp = bp;
    *seg = bseg;
    *tt = bt;
    return true;
}

__device__ __forceinline__ float2 closest_point_rect(float4 r, float2 p) {  // shape.rs:167-185
    bool inside = p.x >= r.x && p.x <= r.z && p.y >= r.y && p.y <= r.w;
    if (!inside) return make_float2(clampf(p.x, r.x, r.z), clampf(p.y, r.y, r.w));
    float dl = p.x - r.x, dr = r.z - p.x, db = p.y - r.y, dt = r.w - p.y;
    if (dl <= dr && dl <= db && dl <= dt) return make_float2(r.x, p.y);
    if (dr <= db && dr <= dt) return make_float2(r.z, p.y);
    if (db <= dt) return make_float2(p.x, r.y);
    return make_float2(p.x, r.w);
}

// closest_point_shape (closest.rs:386-456); lp and the result in group space.
static __device__ bool closest_shape(const DevScene& S, int s, float2 lp, float2* out, int* seg, float* t) {
    const float2 p = shape_local_dist(S, s, lp);
    const int4 si = __ldg(&S.s_info[s]);
    const float4 prm = __ldg(&S.s_params[s]);
    const float* X = S.s_xform + 9 * s;
    *seg = -1;
    *t = 0.0f;
    float2 c;
    if (si.x == K_CIRCLE) {
        float r = fabsf(prm.z);
        float dx = p.x - prm.x, dy = p.y - prm.y;
        float len = len2(dx, dy);
        if (len <= 1.0e-8f)
            c = make_float2(prm.x + r, prm.y);
        else {
            float k = r / len;
            c = make_float2(prm.x + dx * k, prm.y + dy * k);
        }
    } else if (si.x == K_ELLIPSE) {
        c = closest_point_ellipse(prm.x, prm.y, fabsf(prm.z), fabsf(prm.w), p);
    } else if (si.x == K_RECT) {
        c = closest_point_rect(prm, p);
    } else {
        if (si.z < 0) return false;
        const int4 pi = __ldg(&S.p_info[2 * si.z]);
        const int4 pi2 = __ldg(&S.p_info[2 * si.z + 1]);
        if (pi2.y == 0) return false;
        const bool approx = pi2.w & PF_APPROX;
        float best = INF_F, bt = 0.0f;
        float2 bp = make_float2(0.0f, 0.0f);
        int bseg = 0;
        for (int k = 0; k < pi.y; ++k) {
            SegGeom sg;
            load_seg(S, pi.x + k, sg);
            if (cubic_cannot_beat(sg, p, approx, best)) continue;
            CPRes cc = seg_closest(sg, p, approx);
            if (cc.dist < best) {
                best = cc.dist;
                bp = make_float2(cc.cx, cc.cy);
                bseg = k;
                bt = cc.t;
            }
        }
        if (!isfinite(best)) return false;
        c = bp;
        *seg = bseg;
        *t = bt;
    }
    *out = xf9(X, c);
    return true;
}

// compute_distance_bvh (api.rs:138-236) with the brute-force fallback compute_distance (api.rs:36-76).
static __device__ bool compute_distance_group(const DevScene& S, int g, float2 pt, float max_radius, ClosestD* best,
                                       unsigned* status) {
    const int4 gb = __ldg(&S.g_bvh[g]);
    const float* s2c = S.g_s2c + 9 * g;
    const float2 lp = xf9(S.g_c2s + 9 * g, pt);
    if (gb.y == 0) {
        bool have = false;
        for (int k = 0; k < gb.w; ++k) {
            const int s = __ldg(&S.g_shape_list[gb.z + k]);
            float2 lc;
            int seg;
            float t;
            if (!closest_shape(S, s, lp, &lc, &seg, &t)) continue;
            const float2 cl = xf9(s2c, lc);
            const float d = len2(cl.x - pt.x, cl.y - pt.y);
            if (d <= max_radius && (!have || d < best->dist)) {
                *best = ClosestD{s, cl, d, seg, t};
                have = true;
            }
        }
        return have;
    }
    float best_dist = max_radius;
    bool have = false;
    int stk[BVH_STACK];
    int sp = 0;
    stk[sp++] = gb.x;
    int guard = 0;
    while (sp > 0 && guard++ < (1 << 20)) {
        const int n = stk[--sp];
        const int4 m = __ldg(&S.gn_meta[n]);
        if (box_distance(__ldg(&S.gn_bounds[n]), lp) > best_dist) continue;
        if (m.z > 0) {
            for (int k = m.y; k < m.y + m.z; ++k) {
                const int s = __ldg(&S.gl_shapes[k]);
                const int4 si = __ldg(&S.s_info[s]);
                float2 lc;
                int seg = -1;
                float t = 0.0f;
                bool ok;
                if (si.x == K_PATH && si.z >= 0 && __ldg(&S.p_info[2 * si.z].w) > 0) {
                    float2 scp;
                    ok = closest_path_bvh(S, si.z, shape_local_dist(S, s, lp), &scp, &seg, &t, status);
                    if (ok) lc = xf9(S.s_xform + 9 * s, scp);
                } else {
                    ok = closest_shape(S, s, lp, &lc, &seg, &t);
                }
                if (!ok) continue;
                const float2 cl = xf9(s2c, lc);
                const float d = len2(cl.x - pt.x, cl.y - pt.y);
                if (d <= best_dist) {
                    best_dist = d;
                    *best = ClosestD{s, cl, d, seg, t};
                    have = true;
                }
            }
        } else {
            const int l = n + 1, r = m.w;
            const float ld = box_distance(__ldg(&S.gn_bounds[l]), lp);
            const float rd = r >= 0 ? box_distance(__ldg(&S.gn_bounds[r]), lp) : INF_F;
            if (sp + 2 > BVH_STACK) {
                atomicOr(status, ST_BVH_LIMIT);
                break;
            }
            if (ld < rd) {
                if (rd <= best_dist) stk[sp++] = r;
                if (ld <= best_dist) stk[sp++] = l;
            } else {
                if (ld <= best_dist) stk[sp++] = l;
                if (rd <= best_dist) stk[sp++] = r;
            }
        }
    }
    return have;
}

__device__ __forceinline__ float smoothstep1(float d) {  // backward/math.rs:9-12
    float t = clampf((d + 1.0f) * 0.5f, 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float d_smoothstep(float d, float d_ret) {  // backward/math.rs:15-22
    if (d < -1.0f || d > 1.0f) return 0.0f;
    float t = (d + 1.0f) * 0.5f;
    float d_t = d_ret * (6.0f * t - 6.0f * t * t);
    return d_t * 0.5f;
}

// ------------------------------------------------------------------ styled strokes (an extension)
// The crate's prefiltered stroke coverage is round: smoothstep(|d| + sw) - smoothstep(|d| - sw)
// (sampling.rs:240-260).  For a PF_STYLED path whose closest point is a segment end with a
// non-round join or cap (the ends the point-sampled stroke excludes, end_excluded), the
// coverage is smoothstep(s + 2 sw) - smoothstep(s), s the signed distance (canvas space,
// negative inside) to the outer edges of that join or cap region; s = |d| - sw elsewhere
// gives the crate's formula back.  The region is the point-sampled one, built in canvas
// space from the canvas images of the vertex and of the control points that set its
// tangents, with the stroke width as radius (the prefiltered stroke's own units): the bevel
// edge, the two miter edges within the limit, a butt end's flat end, a square cap's three
// outer box edges.  A reversal ends both bodies flat; a straight join (|cross| < 1e-6)
// keeps the round formula.  sd->d: partials with respect to (v, qa, qb) in canvas space and
// sw; ids: the path points of v, qa, qb (-1: unused); q: their shape-space positions.
static __device__ __noinline__ bool styled_end_sd(const DevScene& S, int g, int s, int seg, float t, float2 pt, Dl* sd,
                                                  int* ids, float2* q) {
    const int4 si = __ldg(&S.s_info[s]);
    if (si.x != K_PATH || si.z < 0) return false;
    const float sw = __ldg(&S.s_stroke[s]);
    if (!(sw > 0.0f)) return false;
    const int path = si.z;
    const int4 pi = __ldg(&S.p_info[2 * path]);
    const int4 pi2 = __ldg(&S.p_info[2 * path + 1]);
    const int pflags = pi2.w, off = pi.x, n = pi.y, pc = pi2.y;
    if (seg < 0 || seg >= n || !end_excluded(pflags, seg, n, t)) return false;
    const bool closed = pflags & PF_CLOSED;
    const int join = (pflags >> PF_JOIN_SHIFT) & 3, cap = (pflags >> PF_CAP_SHIFT) & 3;
    const float* X = S.s_xform + 9 * s;
    const float* s2c = S.g_s2c + 9 * g;
    ids[0] = ids[1] = ids[2] = -1;
    const bool at1 = t == 1.0f;
    const bool is_join = closed || (at1 ? seg + 1 < n : seg > 0);
    const Dl R = dl_var(sw, 6);
    DV V, e[4];
    int ne = 1;
    bool fan = false, rect = false;
    if (is_join) {
        const int vb = at1 ? (seg + 1) % n : seg, va = vb > 0 ? vb - 1 : n - 1;
        const float4 a0 = __ldg(&S.seg_p[2 * (off + va)]), a1 = __ldg(&S.seg_p[2 * (off + va) + 1]);
        const float4 b0 = __ldg(&S.seg_p[2 * (off + vb)]), b1 = __ldg(&S.seg_p[2 * (off + vb) + 1]);
        const int sa = seg_dir1_slot(a0, a1), sb = seg_dir0_slot(b0, b1);
        q[0] = make_float2(b0.x, b0.y);
        q[1] = seg_slot(a0, a1, sa);
        q[2] = seg_slot(b0, b1, sb);
        const int4 ma = __ldg(&S.seg_meta[off + va]), mb = __ldg(&S.seg_meta[off + vb]);
        ids[0] = mb.z;
        ids[1] = seg_slot_point(ma, sa, closed, pc);
        ids[2] = seg_slot_point(mb, sb, closed, pc);
        const float2 vc = xf9(s2c, xf9(X, q[0])), ac = xf9(s2c, xf9(X, q[1])), bc = xf9(s2c, xf9(X, q[2]));
        if ((vc.x == ac.x && vc.y == ac.y) || (vc.x == bc.x && vc.y == bc.y)) return false;
        V = DV{dl_var(vc.x, 0), dl_var(vc.y, 1)};
        const DV QA{dl_var(ac.x, 2), dl_var(ac.y, 3)}, QB{dl_var(bc.x, 4), dl_var(bc.y, 5)};
        const DV din = dv_unit(dv_sub(V, QA)), dout = dv_unit(dv_sub(QB, V));
        const Dl cr = din.x * dout.y - din.y * dout.x;
        if (fabsf(cr.v) < 1.0e-6f) {
            if (din.x.v * dout.x.v + din.y.v * dout.y.v > 0.0f) return false;  // straight on: the bodies meet
            const DV np{dl_const(0.0f) - din.y, din.x};                        // a reversal: both end flat at v
            e[0] = dv_sub(V, dv_scale(np, R));
            e[1] = dv_add(V, dv_scale(np, R));
        } else {
            const Dl sg = dl_const(cr.v > 0.0f ? 1.0f : -1.0f);
            e[0] = DV{V.x + R * sg * din.y, V.y - R * sg * din.x};
            const DV b{V.x + R * sg * dout.y, V.y - R * sg * dout.x};
            if (join == JOIN_MITER) {
                const Dl sm = ((b.x - e[0].x) * dout.y - (b.y - e[0].y) * dout.x) / cr;
                const DV m = dv_add(e[0], dv_scale(din, sm));
                const float ml = sqrtf((m.x.v - vc.x) * (m.x.v - vc.x) + (m.y.v - vc.y) * (m.y.v - vc.y));
                if (ml <= __ldg(&S.p_miter[path]) * R.v) e[ne++] = m;
            }
            e[ne] = b;
            fan = true;
        }
    } else {
        const bool start = !at1;
        const int sj = start ? 0 : n - 1;
        const float4 q0 = __ldg(&S.seg_p[2 * (off + sj)]), q1 = __ldg(&S.seg_p[2 * (off + sj) + 1]);
        const int sq = start ? seg_dir0_slot(q0, q1) : seg_dir1_slot(q0, q1);
        const int4 m = __ldg(&S.seg_meta[off + sj]);
        q[0] = start ? make_float2(q0.x, q0.y) : make_float2(q1.z, q1.w);
        q[start ? 2 : 1] = seg_slot(q0, q1, sq);
        ids[0] = seg_slot_point(m, start ? 0 : 3, closed, pc);
        ids[start ? 2 : 1] = seg_slot_point(m, sq, closed, pc);
        const float2 vc = xf9(s2c, xf9(X, q[0])), qc = xf9(s2c, xf9(X, q[start ? 2 : 1]));
        if (vc.x == qc.x && vc.y == qc.y) return false;
        V = DV{dl_var(vc.x, 0), dl_var(vc.y, 1)};
        const DV Q = start ? DV{dl_var(qc.x, 4), dl_var(qc.y, 5)} : DV{dl_var(qc.x, 2), dl_var(qc.y, 3)};
        const DV d = dv_unit(dv_sub(V, Q));  // outward along the end
        const DV np{dl_const(0.0f) - d.y, d.x};
        e[0] = dv_sub(V, dv_scale(np, R));
        if (cap == CAP_SQUARE) {
            e[1] = dv_add(e[0], dv_scale(d, R));
            e[2] = dv_add(dv_add(V, dv_scale(np, R)), dv_scale(d, R));
            e[3] = dv_add(V, dv_scale(np, R));
            ne = 3;
            rect = true;
        } else {
            e[1] = dv_add(V, dv_scale(np, R));
        }
    }
    // squared distance to the closest outer edge e[i] -> e[i + 1]
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
    bool inside = false;
    const float2 v0 = make_float2(V.x.v, V.y.v);
    auto val = [](const DV& a) { return make_float2(a.x.v, a.y.v); };
    if (fan)
        for (int i = 0; i < ne; ++i) inside = inside || in_triangle(pt, v0, val(e[i]), val(e[i + 1]));
    if (rect)
        inside = in_triangle(pt, val(e[0]), val(e[1]), val(e[2])) || in_triangle(pt, val(e[0]), val(e[2]), val(e[3]));
    *sd = inside ? dl_const(0.0f) - dist : dist;
    return true;
}
// A closest point at a segment end of a PF_STYLED path: the only case styled_end_sd can
// change, tested inline so that other strokes make no call.
__device__ __forceinline__ bool maybe_styled_end(const DevScene& S, int s, int seg, float t) {
    if (seg < 0 || !(t == 0.0f || t == 1.0f)) return false;
    const int path = __ldg(&S.s_info[s].z);
    return path >= 0 && (__ldg(&S.p_info[2 * path + 1].w) & PF_STYLED);
}

// One prefiltered fragment (sampling.rs:240-300).
struct PFragD {
    bool hit;
    float4 c;  // paint colour with alpha already scaled by the coverage w
    int shape;
    float dist;  // signed distance used for the coverage
    float2 cp;   // closest point, canvas space
    int seg;     // path segment of the closest point or -1
    float t;
    bool within;
};
// Stroke (which = 0) or fill (which = 1) fragment of group g, through one call
// site each of the closest-point search, the inside test and the paint.
__device__ __forceinline__ PFragD prefilter_frag(const DevScene& S, int g, int which, int paint, int rule, float2 pt,
                                                 unsigned* status) {
    PFragD f;
    f.hit = false;
    ClosestD h;
    const bool have = compute_distance_group(S, g, pt, which == 0 ? INF_F : 1.0f, &h, status);
    float d, w;
    if (which == 0) {
        if (!have) return f;
        const float sw = __ldg(&S.s_stroke[h.shape]);
        d = h.dist;
        Dl sd;
        int ids[3];
        float2 q[3];
        if (maybe_styled_end(S, h.shape, h.seg, h.t) && styled_end_sd(S, g, h.shape, h.seg, h.t, pt, &sd, ids, q))
            w = smoothstep1(sd.v + 2.0f * sw) - smoothstep1(sd.v);
        else
            w = smoothstep1(fabsf(d) + sw) - smoothstep1(fabsf(d) - sw);
    } else {
        const bool inside = group_inside(S, g, xf9(S.g_c2s + 9 * g, pt), rule);
        if (!have && !inside) return f;
        d = have ? h.dist : 1.0f;
        if (!inside) d = -d;
        w = smoothstep1(d);
    }
    if (!(w > 0.0f)) return f;
    f.c = paint_color(S, paint, pt);
    f.c.w *= w;
    f.hit = true;
    f.shape = have ? h.shape : 0;
    f.dist = d;
    f.cp = have ? h.point : make_float2(0.0f, 0.0f);
    f.seg = have ? h.seg : -1;
    f.t = have ? h.t : 0.0f;
    f.within = which == 0 ? true : have;
    return f;
}

// Prefiltered coverage reaches past a group's geometry: smoothstep(d) of a fill is
// non-zero for signed distances above -1 pixel, a stroke's for canvas distances below
// its width + 1 (sampling.rs:240-300 visits every group at every sample).  The scene's
// tile lists bin the point-sampled coverage, whose group boxes carry 0.5 pixel of
// slack only, so the prefiltered kernels bin each tile again, in group order, against
// the group box grown by that reach (stroke widths are those of the group's shapes).
__device__ __forceinline__ bool pf_group_reaches(const DevScene& S, int tile, int g) {
    const int4 gi = __ldg(&S.g_info[g]);
    if (gi.x < 0 && gi.y < 0) return false;
    float reach = 1.0f;
    if (gi.y >= 0) {
        const int4 gb = __ldg(&S.g_bvh[g]);
        for (int k = 0; k < gb.w; ++k)
            reach = fmaxf(reach, 1.0f + fabsf(__ldg(&S.s_stroke[__ldg(&S.g_shape_list[gb.z + k])])));
    }
    reach = reach * 1.001f + 0.01f;
    const float4 b = __ldg(&S.g_bbox[g]);
    const int tx = tile % S.tiles_x, ty = tile / S.tiles_x;
    // edge tiles extend to infinity, as in the scene's binning
    const float x0 = tx == 0 ? -INF_F : (float)(tx * TILE), y0 = ty == 0 ? -INF_F : (float)(ty * TILE);
    const float x1 = tx == S.tiles_x - 1 ? INF_F : (float)((tx + 1) * TILE);
    const float y1 = ty == S.tiles_y - 1 ? INF_F : (float)((ty + 1) * TILE);
    return !(b.z + reach < x0 || b.x - reach > x1 || b.w + reach < y0 || b.y - reach > y1);
}
// Groups [base, base + 256) that reach the tile, in order, into list; returns their
// count.  Called by all 256 threads of the CTA; list is valid until the next call.
__device__ __forceinline__ int pf_bin_chunk(const DevScene& S, int tile, int base, int* list, int* warp_cnt) {
    __syncthreads();  // the previous chunk's list is consumed
    const int g = base + (int)threadIdx.x;
    const bool hit = g < S.num_groups && pf_group_reaches(S, tile, g);
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) warp_cnt[wid] = __popc(m);
    __syncthreads();
    int off = 0, total = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const int c = warp_cnt[w];
        off += w < wid ? c : 0;
        total += c;
    }
    if (hit) list[off + __popc(m & ((1u << lane) - 1u))] = g;
    __syncthreads();
    return total;
}

// ------------------------------------------------------------------ forward
__device__ __forceinline__ void forward_prefilter_body(const DevScene& S, const SampleParams& sp, int tile, int round,
                                                       float* accum, float* wsum, unsigned* status, float* sm) {
    const int ri = S.filter_ri;
    const int HW = TILE + 2 * ri;
    const bool use_sm = ri <= MAX_SMEM_RI;
    const int tx = tile % S.tiles_x, ty = tile / S.tiles_x;
    const int spp = sp.sxn * sp.syn;
    const int s_in_tile = round * 256 + (int)threadIdx.x;
    const int pix = sp.layout ? s_in_tile / spp : (int)threadIdx.x, sub = sp.layout ? s_in_tile % spp : round;
    const int x = tx * TILE + (pix % TILE), y = ty * TILE + (pix / TILE);
    __shared__ int list[256], warp_cnt[8];
    if (use_sm)
        for (int i = threadIdx.x; i < HW * HW * 5; i += blockDim.x) sm[i] = 0.0f;
    const bool valid = x < S.width && y < S.height;
    float2 pt = make_float2(0.0f, 0.0f);
    float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (valid) {
        const int sx = sub % sp.sxn, sy = sub / sp.sxn;
        pt = sample_pos(x, y, sx, sy, sp.sxn, sp.syn, S.width, sp.seed, false);
        acc = background_premul(S, y * S.width + x);
    }
    for (int base = 0; base < S.num_groups; base += 256) {
        const int n = pf_bin_chunk(S, tile, base, list, warp_cnt);  // also orders the smem clear above
        if (!valid) continue;
        for (int e = 0; e < n; ++e) {
            const int g = list[e];
            const int4 gi = __ldg(&S.g_info[g]);
#pragma unroll 1
            for (int which = 0; which < 2; ++which) {
                const int p = which == 0 ? gi.y : gi.x;
                if (p < 0) continue;
                PFragD f = prefilter_frag(S, g, which, p, gi.z, pt, status);
                if (f.hit) over(acc, f.c);
            }
        }
    }
    __syncthreads();  // the splat tile is cleared even without groups
    if (valid) splat_sample(S, x, y, tx, ty, ri, HW, use_sm, pt, acc, sm, accum, wsum);
    if (!use_sm) return;
    __syncthreads();
    flush_splat(S, tx, ty, ri, HW, sm, accum, wsum);
}
// The prefiltered forward kernels and their launchers are compiled in prefilter_fwd.cu
// (DVG_PREFILTER_FORWARD, with the crate's root formulas); everything else here.
#if DVG_PREFILTER_FORWARD
__global__ void __launch_bounds__(256, DVG_MINB_PF_FWD) k_forward_prefilter(DevScene S, SampleParams sp, float* accum, float* wsum,
                                                              unsigned* status) {
    extern __shared__ float sm[];
    forward_prefilter_body(S, sp, sp.tile_base + blockIdx.x, blockIdx.y, accum, wsum, status, sm);
}
__global__ void __launch_bounds__(256, DVG_MINB_PF_FWD) k_forward_prefilter_batch(const BatchEntry* __restrict__ B,
                                                                    const int2* __restrict__ work, int items,
                                                                    int* counter, unsigned* status) {
    extern __shared__ float sm[];
    for_each_item(items, counter, [&](int i) {
        const int2 wk = work[i];  // (scene, tile + tiles * sub-sample round)
        const BatchEntry& E = B[wk.x];
        const int tiles = E.S.tiles_x * E.S.tiles_y;
        forward_prefilter_body(E.S, E.sp, wk.y % tiles, wk.y / tiles, E.accum, E.wsum, status, sm);
    });
}
int launch_forward_prefilter(const DevScene& S, const SampleParams& sp, float* accum, float* wsum, unsigned* status,
                             cudaStream_t stream) {
    const int hw = TILE + 2 * S.filter_ri;
    size_t smem = S.filter_ri <= MAX_SMEM_RI ? (size_t)hw * hw * 5 * sizeof(float) : 0;
    dim3 grid(launch_tiles(S, sp), sp.sxn * sp.syn);
    k_forward_prefilter<<<grid, 256, smem, stream>>>(S, sp, accum, wsum, status);
    return 1;
}
int launch_forward_prefilter_batch(const BatchEntry* B, const int2* work, int items, int* counter, int max_ri,
                                   unsigned* status, cudaStream_t stream) {
    const int hw = TILE + 2 * max_ri;
    size_t smem = max_ri <= MAX_SMEM_RI ? (size_t)hw * hw * 5 * sizeof(float) : 0;
    int grid = items;
    if (counter) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_forward_prefilter_batch, 256, smem);
        grid = std::max(1, std::min(items, std::max(per_sm, 1) * std::max(sms, 1)));
    }
    k_forward_prefilter_batch<<<grid, 256, smem, stream>>>(B, work, items, counter, status);
    return 1;
}
#else

// ------------------------------------------------------------------ distance adjoint (backward/distance.rs)
__device__ __forceinline__ void d_xform_pt(const float* m, float2 p, float2 d_out, float* dm, float2* d_p) {
    float t0 = m[0] * p.x + m[1] * p.y + m[2];
    float t1 = m[3] * p.x + m[4] * p.y + m[5];
    float t2 = m[6] * p.x + m[7] * p.y + m[8];
    float ox = t0 / t2, oy = t1 / t2;
    float d0 = d_out.x / t2, d1 = d_out.y / t2, d2 = -(d_out.x * ox + d_out.y * oy) / t2;
    dm[0] += d0 * p.x;
    dm[1] += d0 * p.y;
    dm[2] += d0;
    dm[3] += d1 * p.x;
    dm[4] += d1 * p.y;
    dm[5] += d1;
    dm[6] += d2 * p.x;
    dm[7] += d2 * p.y;
    dm[8] += d2;
    d_p->x += d0 * m[0] + d1 * m[3] + d2 * m[6];
    d_p->y += d0 * m[1] + d1 * m[4] + d2 * m[7];
}
__device__ __forceinline__ float2 d_length2(float2 v, float d_l) {
    float l = sqrtf(v.x * v.x + v.y * v.y);
    if (l == 0.0f) return make_float2(0.0f, 0.0f);
    float k = 2.0f * (0.5f * d_l / l);
    return make_float2(v.x * k, v.y * k);
}
__device__ __forceinline__ float dot2(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul2(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

static __device__ void add_point_grad(const GradPtrs& G, int po, int pc, bool closed, long idx, float2 d) {
    long i = closed ? idx % pc : idx;
    if (i < pc) {
        add_if(G.d_points + 2 * (po + i), d.x);
        add_if(G.d_points + 2 * (po + i) + 1, d.y);
    }
}
// d_closest_point_path (distance.rs:190-394)
static __device__ void d_closest_point_path(const DevScene& S, const GradPtrs& G, int s, float2 pt, float2 d_cp, int seg,
                                     float min_t, float2* d_pt) {
    const int path = __ldg(&S.s_info[s].z);
    const int4 pi = __ldg(&S.p_info[2 * path]);
    const int4 pi2 = __ldg(&S.p_info[2 * path + 1]);
    const int po = pi2.x, np = pi2.y, co = pi2.z;
    const bool closed = pi2.w & PF_CLOSED;
    if (np == 0) return;
    const int pid = __ldg(&S.seg_meta[pi.x + seg].z);
    auto gp = [&](long idx) { return S.points[po + (closed ? idx % np : (idx < np - 1 ? idx : np - 1))]; };
    const int nc = seg < __ldg(&S.path_cdf_info[s].y) ? S.ncp[co + seg] : 0;
    if (nc == 0) {
        long i0 = pid, i1 = (pid + 1) % np;
        float2 p0 = gp(i0), p1 = gp(i1);
        float2 e = sub2(p1, p0);
        float t = dot2(sub2(pt, p0), e) / dot2(e, e);
        if (t < 0.0f) {
            add_point_grad(G, po, np, closed, i0, d_cp);
        } else if (t > 1.0f) {
            add_point_grad(G, po, np, closed, i1, d_cp);
        } else {
            add_point_grad(G, po, np, closed, i0, mul2(d_cp, 1.0f - t));
            add_point_grad(G, po, np, closed, i1, mul2(d_cp, t));
        }
    } else if (nc == 1) {
        long i0 = pid, i1 = pid + 1, i2 = (pid + 2) % np;
        float2 p0 = gp(i0), p1 = gp(i1), p2 = gp(i2);
        float t = min_t;
        float2 d0 = make_float2(0, 0), d1 = d0, d2 = d0;
        if (t == 0.0f) {
            d0 = add2(d0, d_cp);
        } else if (t == 1.0f) {
            d2 = add2(d2, d_cp);
        } else {
            float2 a = add2(sub2(p0, mul2(p1, 2.0f)), p2);
            float2 b = sub2(p1, p0);
            float2 q = sub2(p0, pt);
            float A = dot2(a, a), B = 3.0f * dot2(a, b), C = 2.0f * dot2(b, b) + dot2(a, q);
            float tt = 1.0f - t;
            float d_tt = 2.0f * tt * dot2(d_cp, p0) + 2.0f * t * dot2(d_cp, p1);
            float d_t = -d_tt + 2.0f * tt * dot2(d_cp, p1) + 2.0f * t * dot2(d_cp, p2);
            d0 = add2(d0, mul2(d_cp, tt * tt));
            d1 = add2(d1, mul2(d_cp, 2.0f * tt * t));
            d2 = add2(d2, mul2(d_cp, t * t));
            float pd = 3.0f * A * t * t + 2.0f * B * t + C;
            if (fabsf(pd) > 1.0e-6f) {
                float dA = -(d_t / pd) * t * t * t, dB = -(d_t / pd) * t * t, dC = -(d_t / pd) * t,
                      dD = -(d_t / pd);
                d0 = add2(d0, add2(add2(add2(add2(mul2(a, 2.0f * dA), mul2(sub2(b, a), 3.0f * dB)),
                                             mul2(mul2(b, -4.0f), dC)),
                                        mul2(add2(q, a), dC)),
                                   mul2(sub2(b, q), 2.0f * dD)));
                d1 = add2(d1, add2(add2(add2(add2(mul2(a, -4.0f * dA), mul2(add2(a, mul2(b, -2.0f)), 3.0f * dB)),
                                             mul2(mul2(b, 4.0f), dC)),
                                        mul2(q, -2.0f * dC)),
                                   mul2(q, dD)));
                d2 = add2(d2, add2(add2(mul2(a, 2.0f * dA), mul2(b, 3.0f * dB)), mul2(q, dC)));
                *d_pt = add2(*d_pt, add2(mul2(a, -dC), mul2(b, dD)));
            }
        }
        add_point_grad(G, po, np, closed, i0, d0);
        add_point_grad(G, po, np, closed, i1, d1);
        add_point_grad(G, po, np, closed, i2, d2);
    } else if (nc == 2) {
        long i0 = pid, i1 = pid + 1, i2 = pid + 2, i3 = (pid + 3) % np;
        float2 p0 = gp(i0), p1 = gp(i1), p2 = gp(i2), p3 = gp(i3);
        float t = min_t;
        float2 d0 = make_float2(0, 0), d1 = d0, d2 = d0, d3 = d0;
        if (t == 0.0f) {
            d0 = add2(d0, d_cp);
        } else if (t == 1.0f) {
            d3 = add2(d3, d_cp);
        } else {
            float2 a = add2(add2(add2(mul2(p0, -1.0f), mul2(p1, 3.0f)), mul2(p2, -3.0f)), p3);
            float2 b = add2(add2(mul2(p0, 3.0f), mul2(p1, -6.0f)), mul2(p2, 3.0f));
            float2 c = add2(mul2(p0, -3.0f), mul2(p1, 3.0f));
            float2 q = sub2(p0, pt);
            float A = 3.0f * dot2(a, a);
            if (fabsf(A) < 1.0e-10f) return;
            float B = 5.0f * dot2(a, b);
            float C = 4.0f * dot2(a, c) + 2.0f * dot2(b, b);
            float D = 3.0f * (dot2(b, c) + dot2(a, q));
            float E = dot2(c, c) + 2.0f * dot2(q, b);
            float F = dot2(q, c);
            B = B / A;
            C = C / A;
            D = D / A;
            E = E / A;
            F = F / A;
            float tt = 1.0f - t;
            float d_tt = 3.0f * tt * tt * dot2(d_cp, p0) + 6.0f * tt * t * dot2(d_cp, p1) +
                         3.0f * t * t * dot2(d_cp, p2);
            float d_t = -d_tt + 3.0f * tt * tt * dot2(d_cp, p1) + 6.0f * tt * t * dot2(d_cp, p2) +
                        3.0f * t * t * dot2(d_cp, p3);
            d0 = add2(d0, mul2(d_cp, tt * tt * tt));
            d1 = add2(d1, mul2(d_cp, 3.0f * tt * tt * t));
            d2 = add2(d2, mul2(d_cp, 3.0f * tt * t * t));
            d3 = add2(d3, mul2(d_cp, t * t * t));
            float pd = 5.0f * t * t * t * t + 4.0f * B * t * t * t + 3.0f * C * t * t + 2.0f * D * t + E;
            if (fabsf(pd) > 1.0e-10f) {
                float dB = -(d_t / pd) * t * t * t * t, dC = -(d_t / pd) * t * t * t, dD = -(d_t / pd) * t * t,
                      dE = -(d_t / pd) * t, dF = -(d_t / pd);
                float dA = -dB * B / A - dC * C / A - dD * D / A - dE * E / A - dF * F / A;
                dB /= A;
                dC /= A;
                dD /= A;
                dE /= A;
                dF /= A;
                d0 = add2(d0, mul2(a, 3.0f * -1.0f * 2.0f * dA));
                d1 = add2(d1, mul2(a, 3.0f * 3.0f * 2.0f * dA));
                d2 = add2(d2, mul2(a, 3.0f * -3.0f * 2.0f * dA));
                d3 = add2(d3, mul2(a, 3.0f * 1.0f * 2.0f * dA));
                d0 = add2(d0, mul2(add2(mul2(b, -1.0f), mul2(a, 3.0f)), 5.0f * dB));
                d1 = add2(d1, mul2(add2(mul2(b, 3.0f), mul2(a, -6.0f)), 5.0f * dB));
                d2 = add2(d2, mul2(add2(mul2(b, -3.0f), mul2(a, 3.0f)), 5.0f * dB));
                d3 = add2(d3, mul2(b, 5.0f * dB));
                d0 = add2(d0, add2(mul2(add2(mul2(c, -1.0f), mul2(a, -3.0f)), 4.0f * dC), mul2(b, 3.0f * 2.0f * dC)));
                d1 = add2(d1, add2(mul2(add2(mul2(c, 3.0f), mul2(a, 3.0f)), 4.0f * dC), mul2(b, -6.0f * 2.0f * dC)));
                d2 = add2(d2, add2(mul2(c, -3.0f * dC * 4.0f), mul2(b, 3.0f * 2.0f * dC)));
                d3 = add2(d3, mul2(c, 4.0f * dC));
                d0 = add2(d0, add2(mul2(add2(mul2(c, 3.0f), mul2(b, -3.0f)), 3.0f * dD), mul2(sub2(a, q), 3.0f * dD)));
                d1 = add2(d1, add2(mul2(add2(mul2(c, -6.0f), mul2(b, 3.0f)), 3.0f * dD), mul2(q, 3.0f * 3.0f * dD)));
                d2 = add2(d2, add2(mul2(c, 3.0f * 3.0f * dD), mul2(q, -3.0f * 3.0f * dD)));
                *d_pt = add2(*d_pt, mul2(a, -1.0f * 3.0f * dD));
                d0 = add2(d0, add2(mul2(c, -3.0f * 2.0f * dE), mul2(add2(b, mul2(q, 3.0f)), 2.0f * dE)));
                d1 = add2(d1, add2(mul2(c, 3.0f * 2.0f * dE), mul2(q, -6.0f * 2.0f * dE)));
                d2 = add2(d2, mul2(q, 3.0f * 2.0f * dE));
                *d_pt = add2(*d_pt, mul2(b, -1.0f * 2.0f * dE));
                d0 = add2(d0, add2(mul2(c, dF), mul2(q, -3.0f * dF)));
                d1 = add2(d1, mul2(q, 3.0f * dF));
                *d_pt = add2(*d_pt, mul2(c, -1.0f * dF));
            }
        }
        add_point_grad(G, po, np, closed, i0, d0);
        add_point_grad(G, po, np, closed, i1, d1);
        add_point_grad(G, po, np, closed, i2, d2);
        add_point_grad(G, po, np, closed, i3, d3);
    }
}
// d_closest_point_ellipse (distance.rs:479-561)
static __device__ void d_closest_point_ellipse(float4 prm, float2 pt, float2 d_cp, float2* dc, float2* dr, float2* d_pt) {
    float rx = fabsf(prm.z), ry = fabsf(prm.w);
    const float eps = 1.0e-6f;
    float lx = pt.x - prm.x, ly = pt.y - prm.y;
    if (rx < eps && ry < eps) {
        *dc = add2(*dc, d_cp);
        return;
    }
    if (rx < eps) {
        float hit = (ly >= -ry && ly <= ry) ? 1.0f : 0.0f;
        *dc = add2(*dc, d_cp);
        d_pt->y += d_cp.y * hit;
        if (ly > ry)
            dr->y += d_cp.y;
        else if (ly < -ry)
            dr->y -= d_cp.y;
        return;
    }
    if (ry < eps) {
        float hit = (lx >= -rx && lx <= rx) ? 1.0f : 0.0f;
        *dc = add2(*dc, d_cp);
        d_pt->x += d_cp.x * hit;
        if (lx > rx)
            dr->x += d_cp.x;
        else if (lx < -rx)
            dr->x -= d_cp.x;
        return;
    }
    float sx = lx < 0.0f ? -1.0f : 1.0f, sy = ly < 0.0f ? -1.0f : 1.0f;
    float x = fabsf(lx), y = fabsf(ly);
    float t = dvg_atan2f(y * rx, x * ry);
    float g_t = 0.0f;
    for (int i = 0; i < 20; ++i) {
        float sn = dvg_sinf(t), cs = dvg_cosf(t);
        float gg = rx * x * sn - ry * y * cs + (ry * ry - rx * rx) * sn * cs;
        g_t = rx * x * cs + ry * y * sn + (ry * ry - rx * rx) * (cs * cs - sn * sn);
        if (fabsf(g_t) < 1.0e-12f) break;
        float nx = clampf(t - gg / g_t, 0.0f, HALF_PI_F);
        if (fabsf(nx - t) < 1.0e-6f) {
            t = nx;
            break;
        }
        t = nx;
    }
    float sn = dvg_sinf(t), cs = dvg_cosf(t);
    float d_t = 0.0f;
    dr->x += d_cp.x * sx * cs;
    d_t += d_cp.x * sx * (-rx * sn);
    dr->y += d_cp.y * sy * sn;
    d_t += d_cp.y * sy * (ry * cs);
    float g_a = x * sn - 2.0f * rx * sn * cs, g_b = -y * cs + 2.0f * ry * sn * cs, g_x = rx * sn, g_y = -ry * cs;
    if (fabsf(g_t) > 1.0e-12f) {
        float inv = -d_t / g_t;
        dr->x += inv * g_a;
        dr->y += inv * g_b;
        float d_x = inv * g_x, d_y = inv * g_y;
        d_pt->x += d_x * sx;
        d_pt->y += d_y * sy;
        dc->x -= d_x * sx;
        dc->y -= d_y * sy;
    }
}
// d_closest_point_rect (distance.rs:397-476)
static __device__ void d_closest_point_rect(float4 r, float2 pt, float2 d_cp, float2* d_min, float2* d_max, float2* d_pt) {
    auto dist_to_seg = [&](float2 p0, float2 p1) {
        float2 e = sub2(p1, p0);
        float t = dot2(sub2(pt, p0), e) / dot2(e, e);
        if (t < 0.0f) return len2(p0.x - pt.x, p0.y - pt.y);
        if (t > 1.0f) return len2(p1.x - pt.x, p1.y - pt.y);
        float2 q = sub2(add2(p0, mul2(e, t)), pt);
        return len2(q.x, q.y);
    };
    float2 lt = make_float2(r.x, r.y), rt = make_float2(r.z, r.y), lb = make_float2(r.x, r.w), rb = make_float2(r.z, r.w);
    int id = 0;
    float md = dist_to_seg(lt, lb);
    float top = dist_to_seg(lt, rt), right = dist_to_seg(rt, rb), bottom = dist_to_seg(lb, rb);
    if (top < md) {
        md = top;
        id = 1;
    }
    if (right < md) {
        md = right;
        id = 2;
    }
    if (bottom < md) {
        md = bottom;
        id = 3;
    }
    float2 a = id == 0 ? lt : (id == 1 ? lt : (id == 2 ? rt : lb));
    float2 b = id == 0 ? lb : (id == 1 ? rt : rb);
    float2 da = make_float2(0, 0), db = make_float2(0, 0);
    float2 e = sub2(b, a);
    float t = dot2(sub2(pt, a), e) / dot2(e, e);
    if (t < 0.0f) {
        da = add2(da, d_cp);
    } else if (t > 1.0f) {
        db = add2(db, d_cp);
    } else {
        da = add2(da, mul2(d_cp, 1.0f - t));
        db = add2(db, mul2(d_cp, t));
        float d_t = dot2(d_cp, e);
        float denom = dot2(e, e);
        float d_num = d_t / denom, d_den = d_t * (-t) / denom;
        *d_pt = add2(*d_pt, mul2(e, d_num));
        db = add2(db, mul2(sub2(pt, a), d_num));
        da = add2(da, mul2(sub2(add2(sub2(a, b), a), pt), d_num));
        db = add2(db, mul2(e, 2.0f * d_den));
        da = add2(da, mul2(sub2(a, b), 2.0f * d_den));
    }
    float2 dlt = make_float2(0, 0), drt = dlt, dlb = dlt, drb = dlt;
    if (id == 0) {
        dlt = da;
        dlb = db;
    } else if (id == 1) {
        dlt = da;
        drt = db;
    } else if (id == 2) {
        drt = da;
        drb = db;
    } else {
        dlb = da;
        drb = db;
    }
    *d_min = add2(*d_min, dlt);
    d_max->x += drt.x;
    d_min->y += drt.y;
    d_min->x += dlb.x;
    d_max->y += dlb.y;
    *d_max = add2(*d_max, drb);
}
// Adjoint of styled_end_sd: d_s times its partials, through the shape and group
// transforms, into the path points, the shape and the group transform; returns d_pt
// (the region moves with its three points, so d/dpt = -(the sum of their partials)).
static __device__ __noinline__ float2 d_styled_end(const DevScene& S, const GradPtrs& G, int g, int s, const Dl& sd,
                                                   float d_s, const int* ids, const float2* q) {
    const float* X = S.s_xform + 9 * s;
    const float* s2c = S.g_s2c + 9 * g;
    const int4 pi2 = __ldg(&S.p_info[2 * __ldg(&S.s_info[s].z) + 1]);
    const int po = pi2.x, pc = pi2.y;
    const bool closed = pi2.w & PF_CLOSED;
    float d_s2c[9] = {0}, d_st[9] = {0};
    float2 sum = make_float2(0.0f, 0.0f);
    for (int j = 0; j < 3; ++j) {
        if (ids[j] < 0) continue;
        const float2 gc = make_float2(d_s * sd.d[2 * j], d_s * sd.d[2 * j + 1]);
        sum = add2(sum, gc);
        const float2 qg = xf9(X, q[j]);
        float2 g_qg = make_float2(0.0f, 0.0f), g_q = g_qg;
        d_xform_pt(s2c, qg, gc, d_s2c, &g_qg);
        d_xform_pt(X, q[j], g_qg, d_st, &g_q);
        add_point_grad(G, po, pc, closed, ids[j], g_q);
    }
    for (int k = 0; k < 9; ++k) {
        add_if(G.d_group_transform + 9 * g + k, d_s2c[k]);
        add_if(G.d_shape_transform + 9 * s + k, d_st[k]);
    }
    return make_float2(-sum.x, -sum.y);
}
// d_compute_distance (distance.rs:50-136): geometry, shape and group transform
// gradients by atomics; returns d_pt (for the translation adjoint).
static __device__ float2 d_compute_distance(const DevScene& S, const GradPtrs& G, int g, int s, float2 pt, float2 cp,
                                     int seg, float seg_t, float d_dist) {
    float dx = pt.x - cp.x, dy = pt.y - cp.y;
    if (dx * dx + dy * dy < 1.0e-10f) return make_float2(0.0f, 0.0f);
    const float* c2s = S.g_c2s + 9 * g;
    const float* s2c = S.g_s2c + 9 * g;
    const float* X = S.s_xform + 9 * s;
    float inv[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (__ldg(&S.s_info[s].y) & SF_INVERTIBLE)
        for (int k = 0; k < 6; ++k) inv[k] = S.s_inv[6 * s + k];
    const float2 lpg = xf9(c2s, pt), lcg = xf9(c2s, cp);
    const float2 lps = xf9(inv, lpg), lcs = xf9(inv, lcg);
    float2 dl = d_length2(make_float2(pt.x - cp.x, pt.y - cp.y), d_dist);
    float2 d_pt = dl;
    float2 d_closest = make_float2(-dl.x, -dl.y);
    float d_s2c[9] = {0}, d_st[9] = {0}, d_sinv[9] = {0}, d_c2s[9] = {0};
    float2 d_lcg = make_float2(0, 0), d_lcs = make_float2(0, 0), d_lps = make_float2(0, 0), d_lpg = make_float2(0, 0);
    d_xform_pt(s2c, lcg, d_closest, d_s2c, &d_lcg);
    d_xform_pt(X, lcs, d_lcg, d_st, &d_lcs);
    // d_closest_point (distance.rs:139-187)
    const int4 si = __ldg(&S.s_info[s]);
    const float4 prm = __ldg(&S.s_params[s]);
    float* dp = G.d_shape_params + 4 * s;
    if (si.x == K_CIRCLE) {
        float2 v = make_float2(lps.x - prm.x, lps.y - prm.y);
        float l = len2(v.x, v.y);
        float2 n = l == 0.0f ? make_float2(0, 0) : make_float2(v.x / l, v.y / l);
        float2 d_center = d_lcs;
        float d_radius = dot2(d_lcs, n);
        float2 d_n = mul2(d_lcs, prm.z);
        float2 d_v = make_float2(0, 0);
        if (l != 0.0f) {  // d_normalize (backward/math.rs:53-63)
            d_v = make_float2(d_n.x / l, d_n.y / l);
            float d_l = -dot2(d_n, n) / l;
            d_v = add2(d_v, d_length2(v, d_l));
        }
        d_center = sub2(d_center, d_v);
        d_lps = add2(d_lps, d_v);
        add_if(dp + 0, d_center.x);
        add_if(dp + 1, d_center.y);
        add_if(dp + 2, d_radius);
    } else if (si.x == K_ELLIPSE) {
        float2 dc = make_float2(0, 0), dr = make_float2(0, 0);
        d_closest_point_ellipse(prm, lps, d_lcs, &dc, &dr, &d_lps);
        add_if(dp + 0, dc.x);
        add_if(dp + 1, dc.y);
        add_if(dp + 2, dr.x);
        add_if(dp + 3, dr.y);
    } else if (si.x == K_RECT) {
        float2 dmn = make_float2(0, 0), dmx = make_float2(0, 0);
        d_closest_point_rect(prm, lps, d_lcs, &dmn, &dmx, &d_lps);
        add_if(dp + 0, dmn.x);
        add_if(dp + 1, dmn.y);
        add_if(dp + 2, dmx.x);
        add_if(dp + 3, dmx.y);
    } else if (si.x == K_PATH && seg >= 0 && si.z >= 0) {
        d_closest_point_path(S, G, s, lps, d_lcs, seg, seg_t, &d_lps);
    }
    d_xform_pt(inv, lpg, d_lps, d_sinv, &d_lpg);
    d_xform_pt(c2s, pt, d_lpg, d_c2s, &d_pt);
    // d_group += d_s2c + (-c2s^T) d_c2s c2s^T ; d_shape += (-inv^T) d_sinv inv^T + d_st
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float cg = 0.0f, cs = 0.0f;
            for (int k = 0; k < 3; ++k) {
                // (-A^T M)[r][k] summed against A^T[k][c] = A[c][k]
                float mg = (-c2s[0 * 3 + r]) * d_c2s[0 * 3 + k] + (-c2s[1 * 3 + r]) * d_c2s[1 * 3 + k] +
                           (-c2s[2 * 3 + r]) * d_c2s[2 * 3 + k];
                float ms = (-inv[0 * 3 + r]) * d_sinv[0 * 3 + k] + (-inv[1 * 3 + r]) * d_sinv[1 * 3 + k] +
                           (-inv[2 * 3 + r]) * d_sinv[2 * 3 + k];
                cg += mg * c2s[3 * c + k];
                cs += ms * inv[3 * c + k];
            }
            add_if(G.d_group_transform + 9 * g + 3 * r + c, (0.0f + d_s2c[3 * r + c]) + cg);
            add_if(G.d_shape_transform + 9 * s + 3 * r + c, (0.0f + cs) + d_st[3 * r + c]);
        }
    return d_pt;
}

// ------------------------------------------------------------------ interior adjoint (sampling.rs:227-482)
constexpr int MAX_PF = 48;
__device__ __forceinline__ void interior_prefilter_body(const DevScene& S, const SampleParams& sp, int tile, int round,
                                                        const float* d_render, const float* wsum, const GradPtrs& G,
                                                        unsigned* status) {
    __shared__ float red[8][6];
    const int tx = tile % S.tiles_x, ty = tile / S.tiles_x;
    const int spp = sp.sxn * sp.syn;
    const int s_in_tile = round * 256 + (int)threadIdx.x;
    const int pix = sp.layout ? s_in_tile / spp : (int)threadIdx.x, sub = sp.layout ? s_in_tile % spp : round;
    const int x = tx * TILE + (pix % TILE), y = ty * TILE + (pix / TILE);
    const bool valid = x < S.width && y < S.height;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __shared__ int list[256], warp_cnt[8];
    const int W = S.width, H = S.height;
    float2 ps = make_float2(0.0f, 0.0f), pt = ps;
    int pixel = 0;
    float4 dcol = make_float4(0, 0, 0, 0), bg = dcol;
    if (valid) {
        const int sx = sub % sp.sxn, sy = sub / sp.sxn;
        ps = sample_pos(x, y, sx, sy, sp.sxn, sp.syn, W, sp.seed, false);
        pt = make_float2((ps.x / (float)W) * (float)W, (ps.y / (float)H) * (float)H);
        pixel = y * W + x;
        bg = background_premul(S, pixel);
        dcol = gather_d_color(S, d_render, wsum, ps);
    }
    // pass 1: fragments with their distance data
    int code[MAX_PF], fshape[MAX_PF], fseg[MAX_PF];
    float tr[MAX_PF], fdist[MAX_PF], fcx[MAX_PF], fcy[MAX_PF], ft[MAX_PF];
    bool fwithin[MAX_PF];
    int nf = 0;
    bool overflow = false;
    float4 acc = bg;
    for (int base = 0; base < S.num_groups; base += 256) {
        const int n = pf_bin_chunk(S, tile, base, list, warp_cnt);
        if (!valid) continue;
        for (int e = 0; e < n; ++e) {
            const int g = list[e];
            const int4 gi = __ldg(&S.g_info[g]);
#pragma unroll 1
            for (int which = 0; which < 2; ++which) {
                const int p = which == 0 ? gi.y : gi.x;
                if (p < 0) continue;
                PFragD f = prefilter_frag(S, g, which, p, gi.z, pt, status);
                if (!f.hit) continue;
                over(acc, f.c);
                if (nf < MAX_PF) {
                    code[nf] = 2 * g + which;
                    tr[nf] = f.c.w;
                    fshape[nf] = f.shape;
                    fdist[nf] = f.dist;
                    fcx[nf] = f.cp.x;
                    fcy[nf] = f.cp.y;
                    fseg[nf] = f.seg;
                    ft[nf] = f.t;
                    fwithin[nf] = f.within;
                } else {
                    overflow = true;
                }
                ++nf;
            }
        }
    }
    if (overflow) {
        atomicOr(status, ST_FRAGMENT_OVERFLOW);
        nf = 0;
    }
    const bool active = valid && !overflow;
    float4 ret = bg;
    float dcr = dcol.x, dcg = dcol.y, dcb = dcol.z, dca = dcol.w;
    if (nf > 0) {
        float fa = acc.w, fr = acc.x, fg = acc.y, fb = acc.z;
        if (fa > 1.0e-6f) {
            float s = 1.0f / fa;
            fr = fr * s;
            fg = fg * s;
            fb = fb * s;
            float dfr = dcr, dfg = dcg, dfb = dcb;
            dcr = dcr * s;
            dcg = dcg * s;
            dcb = dcb * s;
            dca -= (dfr * fr + dfg * fg + dfb * fb) / fa;
        }
        ret = make_float4(fr, fg, fb, fa);
        float run = 1.0f;
        for (int i = nf - 1; i >= 0; --i) {
            float a = tr[i];
            tr[i] = run;
            run = run * (1.0f - a);
        }
        dcol = make_float4(dcr * run, dcg * run, dcb * run, dca * run);
    }
    if (active && S.bg_image) {
        if (G.d_background_image) {
            float* b = G.d_background_image + 4 * (size_t)pixel;
            add_if(b + 0, dcol.x);
            add_if(b + 1, dcol.y);
            add_if(b + 2, dcol.z);
            add_if(b + 3, dcol.w);
        }
        dcol = make_float4(0, 0, 0, 0);
    }
    if (!active) dcol = make_float4(0, 0, 0, 0);
    // pass 3: compositing adjoint with coverage and distance derivatives; the warp
    // visits only entries some lane hit (smallest next fragment code over the warp).
    int cur = 0;
    float4 prev = bg;
    while (true) {
        const int mine = cur < nf ? code[cur] : 0x7fffffff;
        const int nxt = __reduce_min_sync(0xffffffffu, mine);
        if (nxt == 0x7fffffff) break;
        const int g = nxt >> 1, which = nxt & 1;  // code = 2 * group + (0 stroke, 1 fill)
        const int4 gi = __ldg(&S.g_info[g]);
        const int p = which == 0 ? gi.y : gi.x;
        const bool has = mine == nxt;
        {
            float4 dv = make_float4(0, 0, 0, 0);
            int i = cur;
            float w = 0.0f, d_w = 0.0f;
            bool styled = false;
            Dl sd;
            int sids[3];
            float2 sq[3];
            if (has) {
                float4 c = paint_color(S, p, pt);
                const float d = fdist[i];
                if (which == 0) {
                    const float sw = __ldg(&S.s_stroke[fshape[i]]);
                    styled = maybe_styled_end(S, fshape[i], fseg[i], ft[i]) &&
                             styled_end_sd(S, g, fshape[i], fseg[i], ft[i], pt, &sd, sids, sq);
                    w = styled ? smoothstep1(sd.v + 2.0f * sw) - smoothstep1(sd.v)
                               : smoothstep1(fabsf(d) + sw) - smoothstep1(fabsf(d) - sw);
                } else {
                    w = smoothstep1(d);
                }
                c.w *= w;
                const float T = tr[i];
                const float r_ = dcr * T, g_ = dcg * T, b_ = dcb * T, a_ = dca * T;
                float d_alpha = a_ * (1.0f - prev.w);
                d_alpha += r_ * (c.x - prev.x) + g_ * (c.y - prev.y) + b_ * (c.z - prev.z);
                if (w != 0.0f) {
                    d_w = w > 0.0f ? (c.w / w) * d_alpha : 0.0f;
                    dv = make_float4(r_ * c.w, g_ * c.w, b_ * c.w, d_alpha * w);
                }
                over(prev, c);
                ++cur;
            }
            const int kind = __ldg(&S.paint_info[p].x);
            if (kind == P_SOLID) {
                float s0 = warp_sum(dv.x), s1 = warp_sum(dv.y), s2 = warp_sum(dv.z), s3 = warp_sum(dv.w);
                if (lane == 0) {
                    float* d = G.d_paint_params + 4 * p;
                    add_if(d + 0, s0);
                    add_if(d + 1, s1);
                    add_if(d + 2, s2);
                    add_if(d + 3, s3);
                }
            }
            float2 tdelta = make_float2(0.0f, 0.0f);
            if (kind != P_SOLID) d_gradient_paint_warp(S, G, p, pt, dv, has && w != 0.0f, &tdelta);
            if (!has || w == 0.0f) continue;
            const float d = fdist[i];
            float d_d;
            bool geom = true;
            if (which == 0 && styled) {
                const float sw = __ldg(&S.s_stroke[fshape[i]]);
                const float dp = d_smoothstep(sd.v + 2.0f * sw, d_w), dm = d_smoothstep(sd.v, d_w);
                const float d_s = dp - dm;
                add_if(G.d_shape_stroke_width + fshape[i], 2.0f * dp + d_s * sd.d[6]);
                const float2 dpt = d_styled_end(S, G, g, fshape[i], sd, d_s, sids, sq);
                tdelta.x += -dpt.x;
                tdelta.y += -dpt.y;
                d_d = 0.0f;
                geom = false;
            } else if (which == 0) {
                const float sw = __ldg(&S.s_stroke[fshape[i]]);
                const float ap = fabsf(d) + sw, am = fabsf(d) - sw;
                const float dap = d_smoothstep(ap, d_w), dam = -d_smoothstep(am, d_w);
                d_d = dap + dam;
                if (d < 0.0f) d_d = -d_d;
                add_if(G.d_shape_stroke_width + fshape[i], dap - dam);
            } else {
                d_d = d_smoothstep(d, d_w);
                if (d < 0.0f) d_d = -d_d;
                geom = fwithin[i];
            }
            if (fabsf(d_d) > 1.0e-10f && geom) {
                float2 dpt = d_compute_distance(S, G, g, fshape[i], pt, make_float2(fcx[i], fcy[i]), fseg[i], ft[i],
                                                d_d);
                tdelta.x += -dpt.x;
                tdelta.y += -dpt.y;
            }
            if (G.d_translation) {
                add_if(G.d_translation + 2 * (size_t)pixel, tdelta.x);
                add_if(G.d_translation + 2 * (size_t)pixel + 1, tdelta.y);
            }
        }
    }
    float dradius = active ? filter_radius_adjoint(S, d_render, wsum, ps, ret) : 0.0f;
    float v[5] = {dcol.x, dcol.y, dcol.z, dcol.w, dradius};
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
        for (int k = 0; k < 5; ++k) red[wid][k] = v[k];
    __syncthreads();
    if (threadIdx.x < 5) {
        float s = 0.0f;
        for (int w2 = 0; w2 < 8; ++w2) s += red[w2][threadIdx.x];
        if (threadIdx.x < 4)
            add_if(G.d_background + threadIdx.x, s);
        else
            add_if(G.d_filter_radius, s);
    }
}

__global__ void __launch_bounds__(256, DVG_MINB_PF_INT) k_interior_prefilter(DevScene S, SampleParams sp, const float* d_render,
                                                            const float* wsum, GradPtrs G, unsigned* status) {
    interior_prefilter_body(S, sp, sp.tile_base + blockIdx.x, blockIdx.y, d_render, wsum, G, status);
}
__global__ void __launch_bounds__(256, DVG_MINB_PF_INT) k_interior_prefilter_batch(const BatchEntry* __restrict__ B,
                                                                  const int2* __restrict__ work, int items,
                                                                  int* counter, unsigned* status) {
    for_each_item(items, counter, [&](int i) {
        const int2 wk = work[i];  // (scene, tile + tiles * sub-sample round)
        const BatchEntry& E = B[wk.x];
        const int tiles = E.S.tiles_x * E.S.tiles_y;
        interior_prefilter_body(E.S, E.sp, wk.y % tiles, wk.y / tiles, E.d_render, E.wsum, E.G, status);
    });
}

int launch_interior_prefilter(const DevScene& S, const SampleParams& sp, const float* d_render, const float* wsum,
                              const GradPtrs& G, unsigned* status, cudaStream_t stream) {
    dim3 grid(launch_tiles(S, sp), sp.sxn * sp.syn);
    k_interior_prefilter<<<grid, 256, 0, stream>>>(S, sp, d_render, wsum, G, status);
    return 1;
}

int launch_interior_prefilter_batch(const BatchEntry* B, const int2* work, int items, int* counter, unsigned* status,
                                    cudaStream_t stream) {
    int grid = items;
    if (counter) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_interior_prefilter_batch, 256, 0);
        grid = std::max(1, std::min(items, std::max(per_sm, 1) * std::max(sms, 1)));
    }
    k_interior_prefilter_batch<<<grid, 256, 0, stream>>>(B, work, items, counter, status);
    return 1;
}


// ------------------------------------------------------------------ signed distance field
// The closest boundary over all groups (gpu/kernels/sdf.rs:8-115 forward,
// backward/sampling.rs:14-68 backward): groups last to first, each searched with the
// best distance so far as its bound and kept only when strictly closer; `init` is
// the starting bound (1e20 in the crate's forward kernel, infinity in its backward).
// The order matters: inside a group the crate prunes BVH nodes by their distance in
// the group's local frame against that canvas-space bound, so a group whose
// transform enlarges distances can return a different point under a different
// bound; the loop therefore keeps the crate's order.  A group whose conservative
// canvas box is farther than the bound is skipped without its transform (it cannot
// return a point within the bound, which is all the crate's search would accept).
static __device__ bool sdf_closest(const DevScene& S, const float4* g_bbox, float2 pt, float init, ClosestD* best,
                            int* group, unsigned* status) {
    float best_dist = init;
    bool found = false;
    for (int g = S.num_groups - 1; g >= 0; --g) {
        if (box_distance(__ldg(&g_bbox[g]), pt) > best_dist) continue;
        ClosestD h;
        if (compute_distance_group(S, g, pt, best_dist, &h, status) && h.dist < best_dist) {
            best_dist = h.dist;
            *best = h;
            *group = g;
            found = true;
        }
    }
    return found;
}
// Sign from the closest group's fill: negative inside (fill_inside_group / is_inside_bvh).
__device__ __forceinline__ bool sdf_inside(const DevScene& S, int g, float2 pt) {
    const int4 gi = __ldg(&S.g_info[g]);
    return gi.x >= 0 && group_inside(S, g, xf9(S.g_c2s + 9 * g, pt), gi.z);
}
static __device__ float sdf_signed(const DevScene& S, float2 pt, unsigned* status) {
    ClosestD b;
    int g = 0;
    if (!sdf_closest(S, S.g_bbox, pt, 1.0e20f, &b, &g, status)) return 0.0f;
    return sdf_inside(S, g, pt) ? -b.dist : b.dist;
}

// Renderer::render_sdf (gpu/kernels/sdf.rs:118-200): thread = pixel; mean signed
// distance of the pixel's samples at the kernel's positions x + (sx + r) * (1/sx_n).
__global__ void DVG_SDF_BOUNDS k_render_sdf(DevScene S, SampleParams sp, float* out, unsigned* status) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (x >= S.width || y >= S.height) return;
    const float inv_sx = 1.0f / (float)sp.sxn, inv_sy = 1.0f / (float)sp.syn;
    float acc = 0.0f;
    for (int sy = 0; sy < sp.syn; ++sy)
        for (int sx = 0; sx < sp.sxn; ++sx) {
            float rx = 0.5f, ry = 0.5f;
            if (sp.jitter) {
                const uint64_t idx = (((uint64_t)y * S.width + x) * sp.syn + sy) * sp.sxn + sx;
                Pcg32 rng(idx, (uint64_t)sp.seed);
                rx = rng.next_f32();
                ry = rng.next_f32();
            }
            const float2 pt = make_float2((float)x + ((float)sx + rx) * inv_sx, (float)y + ((float)sy + ry) * inv_sy);
            acc += sdf_signed(S, pt, status);
        }
    out[(size_t)y * S.width + x] = acc * (1.0f / (float)(sp.sxn * sp.syn));
}

// Renderer::eval_positions (gpu/kernels/sdf.rs:203-262): thread = point.
__global__ void __launch_bounds__(256) k_eval_positions(DevScene S, const float2* pos, uint64_t n, float* out,
                                                        unsigned* status) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = sdf_signed(S, pos[i], status);
}

// sample_distance (backward/sampling.rs:14-68) at one point with adjoint d_dist.
__device__ __forceinline__ void sdf_adjoint(const DevScene& S, const GradPtrs& G, float2 pt, float d_dist,
                                            int translation_pixel, unsigned* status) {
    ClosestD b;
    int g = 0;
    if (!sdf_closest(S, S.g_bbox, pt, INF_F, &b, &g, status)) return;
    const float d_abs = sdf_inside(S, g, pt) ? -d_dist : d_dist;
    const float2 dpt = d_compute_distance(S, G, g, b.shape, pt, b.point, b.seg, b.t, d_abs);
    if (translation_pixel >= 0 && G.d_translation) {
        add_if(G.d_translation + 2 * (size_t)translation_pixel, -dpt.x);
        add_if(G.d_translation + 2 * (size_t)translation_pixel + 1, -dpt.y);
    }
}

// The d_sdf_image part of render_backward (backward/render.rs:95-188): thread = sample
// at the CPU sample position; every sample passes its pixel's full d_sdf (the crate
// does not divide it by the sample count).
__global__ void DVG_SDF_BOUNDS k_sdf_backward(DevScene S, SampleParams sp, const float* d_sdf, GradPtrs G,
                                                      int translation, unsigned* status) {
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t spp = (uint64_t)sp.sxn * sp.syn;
    if (idx >= (uint64_t)S.width * S.height * spp) return;
    const int sx = (int)(idx % sp.sxn), sy = (int)((idx / sp.sxn) % sp.syn);
    const uint64_t p = idx / spp;
    const int x = (int)(p % S.width), y = (int)(p / S.width);
    const float d = d_sdf[p];
    if (d == 0.0f) return;
    const float2 pt = sample_pos(x, y, sx, sy, sp.sxn, sp.syn, S.width, sp.seed, sp.jitter);
    sdf_adjoint(S, G, pt, d, translation ? (int)p : -1, status);
}

// render_backward_positions (backward/render.rs:213-281): thread = point.
__global__ void DVG_SDF_BOUNDS k_positions_backward(DevScene S, const float2* pos, uint64_t n,
                                                            const float* d_values, GradPtrs G, int translation,
                                                            unsigned* status) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float d = d_values[i];
    if (d == 0.0f) return;
    const float2 pt = pos[i];
    int tp = -1;
    if (translation) {  // translation_index_for_point
        const int x = f2i(pt.x), y = f2i(pt.y);
        if (x >= 0 && y >= 0 && x < S.width && y < S.height) tp = y * S.width + x;
    }
    sdf_adjoint(S, G, pt, d, tp, status);
}

int launch_render_sdf(const DevScene& S, const SampleParams& sp, float* out, unsigned* status, cudaStream_t stream) {
    if (S.width <= 0 || S.height <= 0) return 0;
    dim3 grid((unsigned)((S.width + 15) / 16), (unsigned)((S.height + 15) / 16));
    k_render_sdf<<<grid, 256, 0, stream>>>(S, sp, out, status);
    return 1;
}
int launch_eval_positions(const DevScene& S, const float2* pos, uint64_t n, float* out, unsigned* status,
                          cudaStream_t stream) {
    if (n == 0) return 0;
    k_eval_positions<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(S, pos, n, out, status);
    return 1;
}
int launch_sdf_backward(const DevScene& S, const SampleParams& sp, const float* d_sdf, const GradPtrs& G,
                        bool translation, unsigned* status, cudaStream_t stream) {
    const uint64_t total = (uint64_t)S.width * S.height * sp.sxn * sp.syn;
    if (total == 0) return 0;
    k_sdf_backward<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(S, sp, d_sdf, G, translation ? 1 : 0, status);
    return 1;
}
int launch_positions_backward(const DevScene& S, const float2* pos, uint64_t n, const float* d_values,
                              const GradPtrs& G, bool translation, unsigned* status, cudaStream_t stream) {
    if (n == 0) return 0;
    k_positions_backward<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(S, pos, n, d_values, G,
                                                                          translation ? 1 : 0, status);
    return 1;
}

#endif  // DVG_PREFILTER_FORWARD
}  // namespace dvgb
