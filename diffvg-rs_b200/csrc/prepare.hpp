// prepare.hpp — host-side scene preparation.
//
// Turns a dvg_scene_desc into flat, index-based tables that are uploaded to
// HBM once per scene: per-group transforms and paints, the crate's two-level
// median-split BVH (groups over shapes, paths over segments; same topology as
// src/distance/bvh.rs:149-238 so that the set of evaluated primitives — and
// hence every inside/outside decision — matches the crate), stroke segments
// with their padded bounds, and the boundary-sampling CDF tables
// (src/backward/boundary.rs:46-451).  Replaces prepare_scene /
// prepare_scene_backward (src/renderer/prepare.rs:114-357,
// src/renderer/prepare_backward.rs:45-115), which instead packed AoS f32
// buffers with float-encoded indices.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dvg.h"

namespace dvgb {

struct HostScene {
    uint32_t width = 0, height = 0;
    uint32_t num_groups = 0, num_shapes = 0, num_paints = 0, num_paths = 0;
    uint32_t total_points = 0, total_stops = 0;
    uint32_t filter_type = 0;
    float filter_radius = 0.5f;
    float bg[4] = {0, 0, 0, 0};
    std::vector<float> bg_image;  // empty when none

    // groups
    std::vector<float> g_c2s;          // 9 per group (canvas_to_shape)
    std::vector<float> g_s2c;          // 9 per group
    std::vector<int32_t> g_info;       // 4 per group: fill paint, stroke paint, fill rule, 0
    std::vector<int32_t> g_bvh;        // 4 per group: node offset, node count, shape-list offset, shape-list count
    std::vector<float> g_bbox;         // 4 per group: canvas-space conservative bounds
    std::vector<int32_t> g_shape_list; // flat ShapeGroup::shape_indices (valid ids only)
    // group BVH nodes (global), preorder with skip links
    std::vector<float> gn_bounds;      // 4 per node
    std::vector<int32_t> gn_meta;      // 4 per node: skip, leaf start (into gl_shapes), count, right child
                                       // (absolute indices; left child of an inner node = node + 1; -1 none)
    std::vector<int32_t> gl_shapes;    // leaf order: shape id, per entry

    // shapes
    std::vector<int32_t> s_info;       // 4 per shape: kind, flags, path index (-1), 0
    std::vector<float> s_params;       // 4 per shape
    std::vector<float> s_inv;          // 6 per shape: inverse of Shape::transform (rows 0..1)
    std::vector<float> s_xform;        // 9 per shape
    std::vector<float> s_stroke;       // 1 per shape
    std::vector<float> s_box;          // 4 per shape: padded group-space bounds (the group BVH's leaf boxes)
    std::vector<float> s_padmul;       // 1 per shape: stroke-pad multiplier (miter limit for miter joins,
                                       // at least sqrt 2 for open paths with square caps, else 1)

    // paths (one record per path shape)
    std::vector<int32_t> p_info;       // 8 per path: seg off, seg count, node off, node count,
                                       //             point off, point count, ctrl off, flags
    std::vector<int32_t> p_shape;      // 1 per path: its shape id
    std::vector<float> p_miter;        // 1 per path: miter limit (>= 1) for miter joins
    bool any_styled = false;           // some path has PATH_STYLED
    std::vector<float> pn_bounds;      // 4 per path-BVH node
    std::vector<int32_t> pn_meta;      // 4 per node: skip, leaf start (into pl_segs), count, right child
    std::vector<int32_t> pl_segs;      // leaf order: global segment index
    std::vector<float> seg_p;          // 8 per segment: p0..p3
    std::vector<float> seg_r;          // 4 per segment: r0..r3
    std::vector<int32_t> seg_meta;     // 4 per segment: kind, segment index, point id, shape id
    std::vector<float> points;         // 2 per point (flat, as in the description)
    std::vector<float> thickness;      // 1 per point (0 when absent)
    std::vector<uint8_t> ncp;          // flat num_control_points

    // paints
    std::vector<int32_t> paint_info;   // 4 per paint: kind, stop offset, stop count, 0
    std::vector<float> paint_params;   // 4 per paint
    std::vector<float> stop_offsets;
    std::vector<float> stop_colors;    // 4 per stop

    // boundary sampling tables (src/backward/boundary.rs:46-110)
    bool boundary_ok = false;
    std::vector<float> shape_len;      // per shape
    std::vector<float> bcdf, bpmf;     // over (group, shape) pairs in group order
    std::vector<int32_t> b_shape, b_group;
    std::vector<int32_t> path_cdf_info;  // 4 per shape: cdf offset, count, valid, 0 (a slot for every path,
                                         // so the tables can be rebuilt in place when points move)
    std::vector<float> path_cdf, path_pmf, path_len_arr;
    std::vector<int32_t> path_pid;       // point id per cdf entry
};

// Bits of a path's flags word (the fourth int of its second p_info entry) above the
// DVG_PATH_* bits: set when the stroke uses joins or caps other than round.
enum PathStyle : int32_t {
    PATH_STYLED = 8,
    PATH_JOIN_SHIFT = 4,  // 2 bits: DVG_JOIN_*
    PATH_CAP_SHIFT = 6,   // 2 bits: DVG_CAP_*
};

enum ShapeFlags : int32_t {
    SF_IDENTITY = 1,    // Mat3::is_identity (1e-6 tolerance)
    SF_INVERTIBLE = 2,  // Mat3::inverse succeeded
    SF_HAS_BOUNDS = 4,
};

// Returns DVG_OK or an error status with *err set to the reason.
dvg_status prepare_scene(const dvg_scene_desc* d, HostScene* out, std::string* err);

}  // namespace dvgb
