// prepare.cpp — host-side scene preparation (see prepare.hpp).
//
// Compiled with -ffp-contract=off: the bounds, inverses and CDFs built here
// feed decisions that must match the crate's f32 arithmetic bit for bit.
#include "prepare.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>

namespace dvgb {
namespace {

const float kPi = 3.14159265358979323846f;
const float kInf = std::numeric_limits<float>::infinity();
const size_t kLeafSize = 8;  // BVH_LEAF_SIZE, src/distance/bvh.rs:12
const float kSqrt2Up = 1.41422f;  // sqrt(2) rounded up

uint32_t stroke_join_of(const dvg_scene_desc* d, uint32_t s) {  // validated: <= DVG_JOIN_ROUND
    return d->shape_stroke_join ? d->shape_stroke_join[s] : (uint32_t)DVG_JOIN_ROUND;
}
uint32_t stroke_cap_of(const dvg_scene_desc* d, uint32_t s) {  // validated: <= DVG_CAP_ROUND
    return d->shape_stroke_cap ? d->shape_stroke_cap[s] : (uint32_t)DVG_CAP_ROUND;
}

struct Box {
    float x0, y0, x1, y1;
};
Box empty_box() { return Box{kInf, kInf, -kInf, -kInf}; }
void grow(Box& b, const Box& o) {
    b.x0 = std::fmin(b.x0, o.x0);
    b.y0 = std::fmin(b.y0, o.y0);
    b.x1 = std::fmax(b.x1, o.x1);
    b.y1 = std::fmax(b.y1, o.y1);
}
void grow_pt(Box& b, float x, float y) {
    b.x0 = std::fmin(b.x0, x);
    b.y0 = std::fmin(b.y0, y);
    b.x1 = std::fmax(b.x1, x);
    b.y1 = std::fmax(b.y1, y);
}
Box inflate(Box b, float pad) {  // src/distance/shape.rs:92-99
    pad = std::fmax(pad, 0.0f);
    return Box{b.x0 - pad, b.y0 - pad, b.x1 + pad, b.y1 + pad};
}

struct Affine {  // Mat3 in f32, row-major
    float m[9];
};
void apply(const Affine& t, float x, float y, float* ox, float* oy) {  // src/math.rs:198-202
    *ox = t.m[0] * x + t.m[1] * y + t.m[2];
    *oy = t.m[3] * x + t.m[4] * y + t.m[5];
}
bool is_identity(const Affine& t) {  // src/math.rs:212-222
    const float e = 1.0e-6f;
    return std::fabs(t.m[0] - 1.0f) < e && std::fabs(t.m[1]) < e && std::fabs(t.m[2]) < e &&
           std::fabs(t.m[3]) < e && std::fabs(t.m[4] - 1.0f) < e && std::fabs(t.m[5]) < e &&
           std::fabs(t.m[6]) < e && std::fabs(t.m[7]) < e && std::fabs(t.m[8] - 1.0f) < e;
}
bool inverse(const Affine& t, float inv6[6]) {  // src/math.rs:269-290
    float a = t.m[0], b = t.m[1], c = t.m[3], d = t.m[4], tx = t.m[2], ty = t.m[5];
    float det = a * d - b * c;
    if (std::fabs(det) < 1.0e-6f) return false;
    float id = 1.0f / det;
    float m00 = d * id, m01 = -b * id, m10 = -c * id, m11 = a * id;
    inv6[0] = m00;
    inv6[1] = m01;
    inv6[2] = -(m00 * tx + m01 * ty);
    inv6[3] = m10;
    inv6[4] = m11;
    inv6[5] = -(m10 * tx + m11 * ty);
    return true;
}
float max_scale(const Affine& t) {  // src/math.rs:250-266
    float sx = std::sqrt(t.m[0] * t.m[0] + t.m[3] * t.m[3]);
    float sy = std::sqrt(t.m[1] * t.m[1] + t.m[4] * t.m[4]);
    return std::fmax(sx, sy);
}

// One stroke/fill segment of a path, as src/distance/bvh.rs:130-154 stores it.
struct Seg {
    int kind, index, point_id;
    float p[8];
    float r[4];
    Box bounds;
};

// Preorder median-split BVH (src/distance/bvh.rs:190-238) emitted with skip links.
// One builder serves every path and group of a scene: its arrays keep their capacity
// from one BVH to the next instead of being allocated per BVH.
struct BvhBuilder {
    std::vector<Box> item;                              // item bounds (filled by the caller)
    std::vector<int32_t> idx;                           // item order; leaves are ranges of it
    std::vector<Box> bounds;                            // per node
    std::vector<int32_t> left, right, start, count, skip;
    std::vector<float> cx, cy;                          // item centres: the split keys

    void build() {
        const size_t n = item.size();
        idx.resize(n);
        std::iota(idx.begin(), idx.end(), 0);
        cx.resize(n);
        cy.resize(n);
        for (size_t i = 0; i < n; ++i) {
            cx[i] = (item[i].x0 + item[i].x1) * 0.5f;
            cy[i] = (item[i].y0 + item[i].y1) * 0.5f;
        }
        bounds.clear();
        left.clear();
        right.clear();
        start.clear();
        count.clear();
        if (n) node(0, n);
        // subtree sizes -> skip link = first node after the subtree (preorder layout)
        const size_t nn = bounds.size();
        skip.assign(nn, 1);
        for (size_t k = nn; k-- > 0;) {
            if (left[k] >= 0) skip[k] += skip[left[k]];
            if (right[k] >= 0) skip[k] += skip[right[k]];
        }
        for (size_t k = 0; k < nn; ++k) skip[k] += (int32_t)k;
    }

  private:
    int32_t node(size_t s, size_t e) {
        Box b = empty_box();
        for (size_t i = s; i < e; ++i) grow(b, item[idx[i]]);
        const size_t n = e - s;
        const int32_t id = (int32_t)bounds.size();
        bounds.push_back(b);
        left.push_back(-1);
        right.push_back(-1);
        start.push_back((int32_t)s);
        count.push_back((int32_t)n);
        if (n <= kLeafSize) return id;
        // stable sort of the range by centre along the longer axis: ties keep their order
        const float* key = (b.x1 - b.x0) >= (b.y1 - b.y0) ? cx.data() : cy.data();
        if (n <= 64) {
            for (size_t i = s + 1; i < e; ++i) {
                const int32_t v = idx[i];
                const float kv = key[v];
                size_t j = i;
                for (; j > s && kv < key[idx[j - 1]]; --j) idx[j] = idx[j - 1];
                idx[j] = v;
            }
        } else {
            std::stable_sort(idx.begin() + s, idx.begin() + e, [key](int32_t a, int32_t c) { return key[a] < key[c]; });
        }
        const size_t mid = s + n / 2;
        const int32_t l = node(s, mid);
        const int32_t r = node(mid, e);
        left[id] = l;
        right[id] = r;
        count[id] = 0;
        return id;
    }
};

bool path_point(const dvg_scene_desc* d, uint32_t po, uint32_t pc, bool closed, size_t index, float* x, float* y) {
    if (pc == 0) return false;  // src/path_utils.rs:7-16
    size_t i;
    if (closed)
        i = index % pc;
    else if (index >= pc)
        return false;
    else
        i = index;
    *x = d->points[2 * (po + i)];
    *y = d->points[2 * (po + i) + 1];
    return true;
}
bool path_point_radius(const dvg_scene_desc* d, uint32_t po, uint32_t pc, bool closed, bool thick, size_t index,
                       float def_r, float* x, float* y, float* r) {  // src/path_utils.rs:19-41
    if (!path_point(d, po, pc, closed, index, x, y)) return false;
    size_t i = closed ? index % pc : index;
    *r = (thick && i < pc) ? d->thickness[po + i] * 1.0f : def_r;
    return true;
}

}  // namespace

dvg_status prepare_scene(const dvg_scene_desc* d, HostScene* out, std::string* err) {
    HostScene& h = *out;
    h = HostScene();
    if (!d) {
        *err = "null scene description";
        return DVG_ERR_INVALID_ARGUMENT;
    }
    h.width = d->width;
    h.height = d->height;
    if ((uint64_t)d->width * d->height > (1ull << 31)) {
        *err = "image size overflow";
        return DVG_ERR_INVALID_SCENE;
    }
    if (d->filter_type > DVG_FILTER_GAUSSIAN) {
        *err = "unknown filter type";
        return DVG_ERR_INVALID_SCENE;
    }
    h.filter_type = d->filter_type;
    h.filter_radius = d->filter_radius;
    for (int k = 0; k < 4; ++k) h.bg[k] = d->background[k];
    if (d->background_image)
        h.bg_image.assign(d->background_image, d->background_image + (size_t)d->width * d->height * 4);
    h.num_shapes = d->num_shapes;
    h.num_groups = d->num_groups;
    h.num_paints = d->num_paints;
    h.total_points = d->total_points;
    h.total_stops = d->total_stops;
    if (d->num_shapes && (!d->shape_kind || !d->shape_params || !d->shape_transform || !d->shape_stroke_width)) {
        *err = "missing shape arrays";
        return DVG_ERR_INVALID_ARGUMENT;
    }
    if (d->num_groups && (!d->group_shape_offset || !d->group_shape_count || !d->group_fill_rule ||
                          !d->group_shape_to_canvas || !d->group_canvas_to_shape || !d->group_fill_paint ||
                          !d->group_stroke_paint)) {
        *err = "missing group arrays";
        return DVG_ERR_INVALID_ARGUMENT;
    }
    if (d->num_groups >= (1u << 30)) {  // fragment codes pack 2 * group + stroke/fill into an int
        *err = "too many groups";
        return DVG_ERR_INVALID_SCENE;
    }
    if (d->num_paints && (!d->paint_kind || !d->paint_params)) {
        *err = "missing paint arrays";
        return DVG_ERR_INVALID_ARGUMENT;
    }
    for (uint32_t s = 0; s < d->num_shapes; ++s)
        if ((d->shape_stroke_join && d->shape_stroke_join[s] > (uint32_t)DVG_JOIN_ROUND) ||
            (d->shape_stroke_cap && d->shape_stroke_cap[s] > (uint32_t)DVG_CAP_ROUND)) {
            *err = "invalid stroke join or cap";
            return DVG_ERR_INVALID_SCENE;
        }
    if (d->total_points) h.points.assign(d->points, d->points + 2 * (size_t)d->total_points);
    h.thickness.assign(d->total_points, 0.0f);
    if (d->thickness && d->total_points) h.thickness.assign(d->thickness, d->thickness + d->total_points);
    if (d->total_ctrl) h.ncp.assign(d->num_control_points, d->num_control_points + d->total_ctrl);

    // ---- shapes and paths
    const uint32_t S = d->num_shapes;
    h.s_info.assign(4 * (size_t)S, 0);
    h.s_params.assign(4 * (size_t)S, 0.0f);
    h.s_inv.assign(6 * (size_t)S, 0.0f);
    h.s_xform.assign(9 * (size_t)S, 0.0f);
    h.s_stroke.assign(S, 0.0f);
    h.s_padmul.assign(S, 1.0f);
    std::vector<Box> shape_box(S, empty_box());
    BvhBuilder bvh;          // reused by every path and group BVH below
    std::vector<Seg> segs;   // one path's segments, reused from path to path
    for (uint32_t s = 0; s < S; ++s) {
        uint32_t kind = d->shape_kind[s];
        if (kind > DVG_SHAPE_ELLIPSE) {
            *err = "unknown shape kind";
            return DVG_ERR_INVALID_SCENE;
        }
        Affine t;
        std::memcpy(t.m, d->shape_transform + 9 * (size_t)s, sizeof(t.m));
        std::memcpy(&h.s_xform[9 * (size_t)s], t.m, sizeof(t.m));
        std::memcpy(&h.s_params[4 * (size_t)s], d->shape_params + 4 * (size_t)s, 4 * sizeof(float));
        h.s_stroke[s] = d->shape_stroke_width[s];
        int32_t flags = 0;
        if (is_identity(t)) flags |= SF_IDENTITY;
        float inv6[6] = {1, 0, 0, 0, 1, 0};
        if (inverse(t, inv6)) flags |= SF_INVERTIBLE;
        std::memcpy(&h.s_inv[6 * (size_t)s], inv6, sizeof(inv6));
        const float* prm = d->shape_params + 4 * (size_t)s;
        // Shape bounds in group space (src/distance/shape.rs:9-59), padded by the stroke (62-78).
        bool has_bounds = true;
        Box gb = empty_box();
        if (kind == DVG_SHAPE_CIRCLE || kind == DVG_SHAPE_ELLIPSE) {
            float cx, cy;
            apply(t, prm[0], prm[1], &cx, &cy);
            float rx = std::fabs(prm[2]);
            float ry = kind == DVG_SHAPE_CIRCLE ? rx : std::fabs(prm[3]);
            float ex = std::sqrt((t.m[0] * rx) * (t.m[0] * rx) + (t.m[1] * ry) * (t.m[1] * ry));
            float ey = std::sqrt((t.m[3] * rx) * (t.m[3] * rx) + (t.m[4] * ry) * (t.m[4] * ry));
            gb = Box{cx - ex, cy - ey, cx + ex, cy + ey};
        } else if (kind == DVG_SHAPE_RECT) {
            float xs[4] = {prm[0], prm[2], prm[2], prm[0]}, ys[4] = {prm[1], prm[1], prm[3], prm[3]};
            for (int k = 0; k < 4; ++k) {
                float x, y;
                apply(t, xs[k], ys[k], &x, &y);
                grow_pt(gb, x, y);
            }
        }
        int32_t path_index = -1;
        if (kind == DVG_SHAPE_PATH) {
            if (!d->path_ctrl_offset || !d->path_ctrl_count || !d->path_point_offset || !d->path_point_count ||
                !d->path_flags) {
                *err = "missing path arrays";
                return DVG_ERR_INVALID_ARGUMENT;
            }
            uint32_t co = d->path_ctrl_offset[s], cc = d->path_ctrl_count[s];
            uint32_t po = d->path_point_offset[s], pc = d->path_point_count[s];
            uint32_t fl = d->path_flags[s];
            if ((uint64_t)co + cc > d->total_ctrl || (uint64_t)po + pc > d->total_points) {
                *err = "path data out of range";
                return DVG_ERR_INVALID_SCENE;
            }
            bool closed = fl & DVG_PATH_CLOSED;
            bool thick = (fl & DVG_PATH_HAS_THICKNESS) && d->thickness;
            if (pc == 0) {
                has_bounds = false;
            } else {
                bool ident = is_identity(t);  // src/path_utils.rs:88-104
                for (uint32_t k = 0; k < pc; ++k) {
                    float x = d->points[2 * (po + k)], y = d->points[2 * (po + k) + 1];
                    if (!ident) apply(t, x, y, &x, &y);
                    grow_pt(gb, x, y);
                }
            }
            path_index = (int32_t)(h.p_info.size() / 8);
            h.p_shape.push_back((int32_t)s);
            // Segments in path order (src/distance/bvh.rs:255-364).
            segs.clear();
            size_t pid = 0;
            float dr = d->shape_stroke_width[s];
            for (uint32_t k = 0; k < cc; ++k) {
                int nc = d->num_control_points[co + k];
                if (nc > 2) break;
                int np = nc + 2;
                Seg sg;
                sg.kind = nc;
                sg.index = (int)k;
                sg.point_id = (int)pid;
                bool ok = true;
                for (int q = 0; q < np && ok; ++q)
                    ok = path_point_radius(d, po, pc, closed, thick, pid + q, dr, &sg.p[2 * q], &sg.p[2 * q + 1],
                                           &sg.r[q]);
                if (!ok || pc == 0) break;
                for (int q = np; q < 4; ++q) {  // duplicate the last point (line: p2=p3=p1, quad: p3=p2)
                    sg.p[2 * q] = sg.p[2 * (np - 1)];
                    sg.p[2 * q + 1] = sg.p[2 * (np - 1) + 1];
                    sg.r[q] = sg.r[np - 1];
                }
                float rmax = sg.r[0];
                for (int q = 1; q < np; ++q) rmax = std::fmax(rmax, sg.r[q]);
                Box bb = empty_box();
                for (int q = 0; q < np; ++q) grow_pt(bb, sg.p[2 * q], sg.p[2 * q + 1]);
                sg.bounds = inflate(bb, rmax);
                segs.push_back(sg);
                pid += (size_t)nc + 1;
            }
            int32_t seg_off = (int32_t)(h.seg_meta.size() / 4);
            int32_t node_off = (int32_t)(h.pn_meta.size() / 4);
            int32_t node_cnt = 0;
            if (!segs.empty()) {
                BvhBuilder& bo = bvh;
                bo.item.clear();
                for (const Seg& sg : segs) bo.item.push_back(sg.bounds);
                bo.build();
                int32_t leaf_base = (int32_t)h.pl_segs.size();
                for (int32_t i : bo.idx) h.pl_segs.push_back(seg_off + i);
                for (size_t n = 0; n < bo.bounds.size(); ++n) {
                    const Box& b = bo.bounds[n];
                    h.pn_bounds.insert(h.pn_bounds.end(), {b.x0, b.y0, b.x1, b.y1});
                    h.pn_meta.insert(h.pn_meta.end(), {node_off + bo.skip[n], leaf_base + bo.start[n], bo.count[n],
                                                       bo.right[n] >= 0 ? node_off + bo.right[n] : -1});
                }
                node_cnt = (int32_t)bo.bounds.size();
                for (const Seg& sg : segs) {
                    h.seg_p.insert(h.seg_p.end(), sg.p, sg.p + 8);
                    h.seg_r.insert(h.seg_r.end(), sg.r, sg.r + 4);
                    h.seg_meta.insert(h.seg_meta.end(), {sg.kind, sg.index, sg.point_id, (int32_t)s});
                }
            }
            int32_t pflags = (int32_t)((closed ? DVG_PATH_CLOSED : 0) | (fl & DVG_PATH_DISTANCE_APPROX) |
                                       (thick ? DVG_PATH_HAS_THICKNESS : 0));
            // Stroke joins / caps other than round (an extension: the crate strokes round only).
            const uint32_t join = stroke_join_of(d, s), cap = stroke_cap_of(d, s);
            if (join != DVG_JOIN_ROUND || (!closed && cap != DVG_CAP_ROUND)) {
                pflags |= PATH_STYLED | (int32_t)(join << PATH_JOIN_SHIFT) | (int32_t)(cap << PATH_CAP_SHIFT);
                h.any_styled = true;
            }
            h.p_miter.push_back(std::fmax(d->shape_miter_limit ? d->shape_miter_limit[s] : 4.0f, 1.0f));
            h.p_info.insert(h.p_info.end(), {seg_off, (int32_t)segs.size(), node_off, node_cnt, (int32_t)po,
                                             (int32_t)pc, (int32_t)co, pflags});
            h.num_paths++;
        }
        if (has_bounds) {
            // max_stroke_radius (src/distance/shape.rs:62-78)
            float scale = std::fmax(max_scale(t), 0.0f);
            float rad = std::fabs(d->shape_stroke_width[s]) * scale;
            if (kind == DVG_SHAPE_PATH && (d->path_flags[s] & DVG_PATH_HAS_THICKNESS) && d->thickness) {
                float mt = 0.0f;
                uint32_t po = d->path_point_offset[s], pc = d->path_point_count[s];
                for (uint32_t k = 0; k < pc; ++k) mt = std::fmax(mt, std::fabs(d->thickness[po + k]));
                rad = std::fmax(rad, mt * scale);
            }
            uint32_t join = stroke_join_of(d, s);
            float miter = d->shape_miter_limit ? d->shape_miter_limit[s] : 4.0f;
            if (join == DVG_JOIN_MITER) h.s_padmul[s] = std::fmax(miter, 1.0f);
            // a square cap's corners lie sqrt(2) radii from the end point
            if (kind == DVG_SHAPE_PATH && !(d->path_flags[s] & DVG_PATH_CLOSED) && stroke_cap_of(d, s) == DVG_CAP_SQUARE)
                h.s_padmul[s] = std::fmax(h.s_padmul[s], kSqrt2Up);
            if (rad > 0.0f) rad *= h.s_padmul[s];
            shape_box[s] = inflate(gb, rad);
            flags |= SF_HAS_BOUNDS;
        }
        h.s_info[4 * (size_t)s] = (int32_t)kind;
        h.s_info[4 * (size_t)s + 1] = flags;
        h.s_info[4 * (size_t)s + 2] = path_index;
    }

    h.s_box.assign(4 * (size_t)S, 0.0f);
    for (uint32_t s = 0; s < S; ++s) {
        const Box& b = shape_box[s];
        float* o = &h.s_box[4 * (size_t)s];
        o[0] = b.x0;
        o[1] = b.y0;
        o[2] = b.x1;
        o[3] = b.y1;
    }

    // ---- paints
    h.paint_info.assign(4 * (size_t)d->num_paints, 0);
    h.paint_params.assign(4 * (size_t)d->num_paints, 0.0f);
    for (uint32_t p = 0; p < d->num_paints; ++p) {
        uint32_t kind = d->paint_kind[p];
        if (kind < DVG_PAINT_SOLID || kind > DVG_PAINT_RADIAL) {
            *err = "unknown paint kind";
            return DVG_ERR_INVALID_SCENE;
        }
        uint32_t so = d->paint_stop_offset ? d->paint_stop_offset[p] : 0;
        uint32_t sc = d->paint_stop_count ? d->paint_stop_count[p] : 0;
        if (kind == DVG_PAINT_SOLID) sc = 0;
        if ((uint64_t)so + sc > d->total_stops) {
            *err = "paint stops out of range";
            return DVG_ERR_INVALID_SCENE;
        }
        h.paint_info[4 * (size_t)p] = (int32_t)kind;
        h.paint_info[4 * (size_t)p + 1] = (int32_t)so;
        h.paint_info[4 * (size_t)p + 2] = (int32_t)sc;
        std::memcpy(&h.paint_params[4 * (size_t)p], d->paint_params + 4 * (size_t)p, 4 * sizeof(float));
    }
    if (d->total_stops) {
        h.stop_offsets.assign(d->stop_offsets, d->stop_offsets + d->total_stops);
        h.stop_colors.assign(d->stop_colors, d->stop_colors + 4 * (size_t)d->total_stops);
    }

    // ---- groups
    const uint32_t G = d->num_groups;
    h.g_c2s.assign(9 * (size_t)G, 0.0f);
    h.g_s2c.assign(9 * (size_t)G, 0.0f);
    h.g_info.assign(4 * (size_t)G, 0);
    h.g_bvh.assign(4 * (size_t)G, 0);
    h.g_bbox.assign(4 * (size_t)G, 0.0f);
    for (uint32_t g = 0; g < G; ++g) {
        uint32_t so = d->group_shape_offset[g], sc = d->group_shape_count[g];
        if ((uint64_t)so + sc > d->total_group_shapes) {
            *err = "group shape list out of range";
            return DVG_ERR_INVALID_SCENE;
        }
        int32_t fp = d->group_fill_paint[g], sp = d->group_stroke_paint[g];
        if (fp >= (int32_t)d->num_paints || sp >= (int32_t)d->num_paints || fp < -1 || sp < -1) {
            *err = "group references invalid paint index";
            return DVG_ERR_INVALID_SCENE;
        }
        std::memcpy(&h.g_c2s[9 * (size_t)g], d->group_canvas_to_shape + 9 * (size_t)g, 9 * sizeof(float));
        std::memcpy(&h.g_s2c[9 * (size_t)g], d->group_shape_to_canvas + 9 * (size_t)g, 9 * sizeof(float));
        h.g_info[4 * (size_t)g] = fp;
        h.g_info[4 * (size_t)g + 1] = sp;
        h.g_info[4 * (size_t)g + 2] = (int32_t)d->group_fill_rule[g];
        int32_t list_off = (int32_t)h.g_shape_list.size();
        std::vector<int32_t> with_bounds;
        for (uint32_t k = 0; k < sc; ++k) {
            uint32_t sid = d->group_shape_ids[so + k];
            if (sid >= S) {  // src/renderer/prepare.rs:175-178
                *err = "group references invalid shape index";
                return DVG_ERR_INVALID_SCENE;
            }
            h.g_shape_list.push_back((int32_t)sid);
            if (h.s_info[4 * (size_t)sid + 1] & SF_HAS_BOUNDS) with_bounds.push_back((int32_t)sid);
        }
        int32_t node_off = (int32_t)(h.gn_meta.size() / 4), node_cnt = 0;
        Box root = empty_box();
        if (!with_bounds.empty()) {  // GroupBvh::build (src/distance/bvh.rs:156-187)
            BvhBuilder& bo = bvh;
            bo.item.clear();
            for (int32_t sid : with_bounds) bo.item.push_back(shape_box[sid]);
            bo.build();
            int32_t leaf_base = (int32_t)h.gl_shapes.size();
            for (int32_t i : bo.idx) h.gl_shapes.push_back(with_bounds[i]);
            for (size_t n = 0; n < bo.bounds.size(); ++n) {
                const Box& b = bo.bounds[n];
                h.gn_bounds.insert(h.gn_bounds.end(), {b.x0, b.y0, b.x1, b.y1});
                h.gn_meta.insert(h.gn_meta.end(), {node_off + bo.skip[n], leaf_base + bo.start[n], bo.count[n],
                                                   bo.right[n] >= 0 ? node_off + bo.right[n] : -1});
            }
            node_cnt = (int32_t)bo.bounds.size();
            root = bo.bounds[0];
        }
        h.g_bvh[4 * (size_t)g] = node_off;
        h.g_bvh[4 * (size_t)g + 1] = node_cnt;
        h.g_bvh[4 * (size_t)g + 2] = list_off;
        h.g_bvh[4 * (size_t)g + 3] = (int32_t)sc;
        // Conservative canvas-space bounds of the group-space root box, for tile binning.
        float* bb = &h.g_bbox[4 * (size_t)g];
        if (node_cnt == 0) {
            bb[0] = bb[1] = kInf;  // nothing can render: empty box
            bb[2] = bb[3] = -kInf;
        } else {
            const float* c = d->group_canvas_to_shape + 9 * (size_t)g;
            double a = c[0], b = c[1], cc = c[3], dd = c[4], tx = c[2], ty = c[5];
            double det = a * dd - b * cc;
            bool finite_root = std::isfinite(root.x0) && std::isfinite(root.y0) && std::isfinite(root.x1) &&
                               std::isfinite(root.y1);
            if (std::fabs(det) < 1e-12 || !finite_root) {
                bb[0] = bb[1] = -kInf;
                bb[2] = bb[3] = kInf;
            } else {
                double xs[4] = {root.x0, root.x1, root.x1, root.x0}, ys[4] = {root.y0, root.y0, root.y1, root.y1};
                double mnx = 1e300, mny = 1e300, mxx = -1e300, mxy = -1e300;
                for (int k = 0; k < 4; ++k) {
                    double lx = xs[k] - tx, ly = ys[k] - ty;
                    double X = (dd * lx - b * ly) / det, Y = (-cc * lx + a * ly) / det;
                    mnx = std::min(mnx, X);
                    mny = std::min(mny, Y);
                    mxx = std::max(mxx, X);
                    mxy = std::max(mxy, Y);
                }
                double pad = 0.5 + 1e-4 * (std::fabs(mnx) + std::fabs(mny) + std::fabs(mxx) + std::fabs(mxy));
                bb[0] = (float)(mnx - pad);
                bb[1] = (float)(mny - pad);
                bb[2] = (float)(mxx + pad);
                bb[3] = (float)(mxy + pad);
            }
        }
    }

    // ---- boundary-sampling tables (src/backward/boundary.rs:46-451)
    h.shape_len.assign(S, 0.0f);
    auto seg_len = [&](uint32_t po, uint32_t pc, bool closed, size_t pid, int nc, bool* ok) -> float {
        float q[8];
        int np = nc + 2;
        *ok = true;
        for (int k = 0; k < np; ++k)
            if (!path_point(d, po, pc, closed, pid + k, &q[2 * k], &q[2 * k + 1])) {
                *ok = false;
                return 0.0f;
            }
        auto L = [](float x0, float y0, float x1, float y1) {
            float dx = x1 - x0, dy = y1 - y0;
            return std::sqrt(dx * dx + dy * dy);
        };
        if (nc == 0) return L(q[0], q[1], q[2], q[3]);
        if (nc == 1) {
            float t = 0.5f, tt = 1.0f - t;
            float vx = q[0] * (tt * tt) + q[2] * (2.0f * tt * t) + q[4] * (t * t);
            float vy = q[1] * (tt * tt) + q[3] * (2.0f * tt * t) + q[5] * (t * t);
            return L(q[0], q[1], vx, vy) + L(vx, vy, q[4], q[5]);
        }
        float v[4];
        for (int k = 0; k < 2; ++k) {
            float t = k == 0 ? 1.0f / 3.0f : 2.0f / 3.0f, tt = 1.0f - t;
            v[2 * k] = q[0] * (tt * tt * tt) + q[2] * (3.0f * tt * tt * t) + q[4] * (3.0f * tt * t * t) +
                       q[6] * (t * t * t);
            v[2 * k + 1] = q[1] * (tt * tt * tt) + q[3] * (3.0f * tt * tt * t) + q[5] * (3.0f * tt * t * t) +
                           q[7] * (t * t * t);
        }
        return L(q[0], q[1], v[0], v[1]) + L(v[0], v[1], v[2], v[3]) + L(v[2], v[3], q[6], q[7]);
    };
    for (uint32_t s = 0; s < S; ++s) {  // compute_shape_lengths (boundary.rs:200-227)
        const float* prm = d->shape_params + 4 * (size_t)s;
        uint32_t kind = d->shape_kind[s];
        float l = 0.0f;
        if (kind == DVG_SHAPE_CIRCLE) {
            l = 2.0f * kPi * std::fabs(prm[2]);
        } else if (kind == DVG_SHAPE_ELLIPSE) {
            float a = std::fabs(prm[2]), b = std::fabs(prm[3]);
            l = (a == 0.0f || b == 0.0f) ? 0.0f : kPi * (3.0f * (a + b) - std::sqrt((3.0f * a + b) * (a + 3.0f * b)));
        } else if (kind == DVG_SHAPE_RECT) {
            l = 2.0f * (std::fabs(prm[2] - prm[0]) + std::fabs(prm[3] - prm[1]));
        } else {
            uint32_t co = d->path_ctrl_offset[s], cc = d->path_ctrl_count[s];
            uint32_t po = d->path_point_offset[s], pc = d->path_point_count[s];
            bool closed = d->path_flags[s] & DVG_PATH_CLOSED;
            if (pc > 0) {
                size_t pid = 0;
                for (uint32_t k = 0; k < cc; ++k) {  // path_length (boundary.rs:230-309)
                    int nc = d->num_control_points[co + k];
                    if (nc > 2) break;
                    bool ok;
                    float sl = seg_len(po, pc, closed, pid, nc, &ok);
                    if (!ok) break;
                    l += sl;
                    pid += (size_t)nc + 1;
                }
            }
        }
        h.shape_len[s] = l;
    }
    float accum = 0.0f;  // build_shape_cdf (boundary.rs:312-346)
    for (uint32_t g = 0; g < G; ++g) {
        uint32_t so = d->group_shape_offset[g], sc = d->group_shape_count[g];
        for (uint32_t k = 0; k < sc; ++k) {
            uint32_t sid = d->group_shape_ids[so + k];
            float l = h.shape_len[sid];
            h.b_shape.push_back((int32_t)sid);
            h.b_group.push_back((int32_t)g);
            accum += l;
            h.bcdf.push_back(accum);
            h.bpmf.push_back(l);
        }
    }
    h.boundary_ok = G > 0 && accum > 0.0f && std::isfinite(accum) && !h.bcdf.empty();
    if (h.boundary_ok) {
        for (float& v : h.bcdf) v /= accum;
        for (float& v : h.bpmf) v /= accum;
    }
    h.path_cdf_info.assign(4 * (size_t)S, 0);
    h.path_len_arr.assign(S, 0.0f);
    for (uint32_t s = 0; s < S; ++s) {  // build_path_cdfs (boundary.rs:349-451)
        if (d->shape_kind[s] != DVG_SHAPE_PATH) continue;
        float l = h.shape_len[s];
        uint32_t co = d->path_ctrl_offset[s], cc = d->path_ctrl_count[s];
        if (cc == 0) continue;
        const bool valid = l > 0.0f && std::isfinite(l);
        uint32_t po = d->path_point_offset[s], pc = d->path_point_count[s];
        bool closed = d->path_flags[s] & DVG_PATH_CLOSED;
        float inv_length = valid ? 1.0f / l : 0.0f;
        int32_t off = (int32_t)h.path_cdf.size();
        size_t pid = 0;
        float prev = 0.0f;
        bool first = true;
        for (uint32_t k = 0; k < cc; ++k) {
            int nc = d->num_control_points[co + k];
            h.path_pid.push_back((int32_t)pid);
            float sl = 0.0f;
            if (nc <= 2) {
                bool ok;
                sl = seg_len(po, pc, closed, pid, nc, &ok);
                if (!ok) sl = 0.0f;
                pid += (size_t)nc + 1;
            }
            float sn = sl * inv_length;
            h.path_pmf.push_back(sn);
            float acc = sn + (first ? 0.0f : prev);
            h.path_cdf.push_back(acc);
            prev = acc;
            first = false;
        }
        h.path_cdf_info[4 * (size_t)s] = off;
        h.path_cdf_info[4 * (size_t)s + 1] = (int32_t)cc;
        h.path_cdf_info[4 * (size_t)s + 2] = valid ? 1 : 0;
        h.path_len_arr[s] = valid ? l : 0.0f;
    }
    return DVG_OK;
}

}  // namespace dvgb
