/*
 * oracle.h — CPU oracle for the diffvg render / backward hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a restatement, in C++, of the diffvg-rs
 * crate's CPU arithmetic (the .rs files under src/backward and src/distance,
 * src/geometry.rs, src/math.rs, src/renderer/rng.rs) and of its GPU forward
 * image pipeline (src/gpu/kernels/forward.rs splat + resolve).  It is linked
 * only by the tests, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline / reference arm — never by the product library.
 *
 * Parity status: pinned against the crate's own known-answer tests
 * (src/distance/tests.rs:7-136, src/geometry.rs:509-519).  Render and
 * gradient outputs are otherwise "parity unpinned": the crate has no tests
 * for them and cannot be built here (no Rust toolchain, no graphics stack).
 */
#ifndef DVG_ORACLE_H
#define DVG_ORACLE_H

#include "../include/dvg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Forward image with the crate's GPU pipeline semantics (weights -> splat -> resolve). */
int oracle_render(const dvg_scene_desc* desc, const dvg_render_options* opts, float* out_rgba);
/* The same image restricted to pixels [x0,x1) x [y0,y1) (out: (x1-x0)*(y1-y0)*4 floats,
 * row-major over the window), bit-identical to those pixels of oracle_render; the
 * per-sample colours run on `threads` host threads. */
int oracle_render_window(const dvg_scene_desc* desc, const dvg_render_options* opts, uint32_t x0, uint32_t y0,
                         uint32_t x1, uint32_t y1, int threads, float* out_rgba);

/* Per-sample premultiplied colour at canvas point (px,py) (eval_scene semantics). */
int oracle_sample_premultiplied(const dvg_scene_desc* desc, const dvg_render_options* opts,
                                float px, float py, float* out4);

/* The image render_backward differentiates (per-sample un-premultiplied colours,
 * filter-weighted per pixel); test infrastructure for finite differences. */
int oracle_render_differentiated(const dvg_scene_desc* desc, const dvg_render_options* opts, float* out);

/* Signed distance field (Renderer::render_sdf, src/renderer/renderer.rs:586), per-point
 * signed distances (Renderer::eval_positions, :719), the d_sdf part of render_backward
 * (src/backward/render.rs:171-188) and render_backward_positions (:213-265). */
int oracle_render_sdf(const dvg_scene_desc* desc, const dvg_render_options* opts, float* out);
int oracle_eval_positions(const dvg_scene_desc* desc, const float* positions, uint64_t n, float* out);
int oracle_sdf_backward(const dvg_scene_desc* desc, const dvg_render_options* opts,
                        const dvg_backward_options* bopts, const float* d_sdf, dvg_grads* grads);
int oracle_positions_backward(const dvg_scene_desc* desc, const dvg_backward_options* bopts,
                              const float* positions, uint64_t n, const float* d_values, dvg_grads* grads);

/* CPU twin of the library's linear BVH build (same outputs as dvg_lbvh_build). */
int oracle_lbvh_build(const float* boxes, uint32_t count, uint64_t* keys_out, int32_t* children_out,
                      float* bounds_out);

/* The crate's CPU render_backward (src/backward/render.rs:35-210).  grads are host
 * buffers that are overwritten (NULL parts skipped, sizes as in dvg.h).  bopts->rng
 * selects the boundary generator (PCG32 as the crate, or Philox4x32-10). */
int oracle_render_backward(const dvg_scene_desc* desc, const dvg_render_options* opts,
                           const dvg_backward_options* bopts, const float* d_render,
                           dvg_grads* grads);

/* Same, with the interior (per-sample) pass and the boundary pass selectable:
 * passes bit0 = interior, bit1 = boundary; threads > 1 runs the sample loops on
 * that many host threads with per-thread gradient buffers. */
int oracle_render_backward_ex(const dvg_scene_desc* desc, const dvg_render_options* opts,
                              const dvg_backward_options* bopts, const float* d_render,
                              dvg_grads* grads, int passes, int threads,
                              unsigned long long sample_begin, unsigned long long sample_end);

/* Deterministic expectation of the boundary pass over boundary seeds (no interior
 * pass): the edge term at the midpoints of m equal steps of every shape's boundary
 * parameter, weighted by the shape's pmf and the crate's sample count.  offset: the
 * colour-sampling offset along the normal in normalised canvas units (1e-4 in the
 * crate, boundary.rs:880-902).  Test infrastructure for the boundary estimators. */
int oracle_boundary_integral(const dvg_scene_desc* desc, const dvg_render_options* opts,
                             const float* d_render, uint32_t m, float offset, int threads,
                             dvg_grads* grads);

/* Weight image (build_weight_image, src/backward/filters.rs:11-67). */
int oracle_weight_image(const dvg_scene_desc* desc, const dvg_render_options* opts, float* out_w);

/* Distance API (src/distance/api.rs) used by the crate's known-answer tests.
 * Returns 1 and fills out (shape_index, point.x, point.y, distance) when a hit exists. */
int oracle_compute_distance(const dvg_scene_desc* desc, uint32_t group, float px, float py,
                            float max_radius, int use_bvh, float* out4);
int oracle_within_distance(const dvg_scene_desc* desc, uint32_t group, float px, float py,
                           int use_bvh);
int oracle_is_inside(const dvg_scene_desc* desc, uint32_t group, float px, float py, int use_bvh);

/* Path::flatten (src/geometry.rs:206-212) of shape `shape`; writes up to cap segments
 * as (x0,y0,x1,y1) and returns the number of segments. */
int oracle_flatten(const dvg_scene_desc* desc, uint32_t shape, float tolerance, float* out,
                   int cap);

/* PCG32 (src/renderer/rng.rs:16-43): first n floats of Pcg32::new(idx, seed). */
void oracle_pcg32_floats(unsigned long long idx, unsigned long long seed, int n, float* out);
/* Philox4x32-10 floats for sample idx / seed (the boundary generator alternative). */
void oracle_philox_floats(unsigned long long idx, unsigned int seed, float* out2);

/* Reference median-split BVH (src/distance/bvh.rs:149-238) of one path shape:
 * writes per node (min.x,min.y,max.x,max.y,left,right,start,count) into nodes
 * (8 floats each, ints stored as floats) and the leaf index order into indices. */
int oracle_path_bvh(const dvg_scene_desc* desc, uint32_t shape, float* nodes, int node_cap,
                    int* indices, int index_cap, int* num_indices);

/* Bounded-sample CPU forward + backward (timing workload): `count` samples spread
 * evenly over the sample sequence plus the proportional share of boundary samples,
 * on `threads` threads; times[0] = set-up seconds, times[1] = sample-loop seconds. */
unsigned long long oracle_fwd_bwd_sample(const dvg_scene_desc* desc, const dvg_render_options* opts,
                                         const dvg_backward_options* bopts, const float* d_render,
                                         unsigned long long count, int threads, double* times);

/* Work of one forward pass for the compute roofline: counts[12] tests reached by the
 * crate's BVH queries without early exits (kinds 0-2 fill line / quadratic / cubic
 * segment, 3-5 stroke segment, 6-8 fill circle / ellipse / rect, 9-11 stroke circle /
 * ellipse / rect) and flops[12] the floating-point operations of those tests in the
 * crate's arithmetic.  Only the counting build (liboracle_ops.so) counts; the oracle
 * proper returns -1. */
int oracle_count_work(const dvg_scene_desc* desc, const dvg_render_options* opts, int threads,
                      unsigned long long* counts, unsigned long long* flops);

#ifdef __cplusplus
}
#endif
#endif
