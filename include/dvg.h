/*
 * dvg.h — C ABI of the B200-native differentiable vector-graphics rasteriser.
 *
 * This is the drop-in boundary for the render / backward hot path of the
 * diffvg-rs crate.  Every entry point takes plain pointers and sizes; no
 * torch or C++ types cross it.  Each declaration names the reference
 * interface it replaces (file:line inside the diffvg-rs crate).
 *
 * Conventions
 *   - A scene is described by dvg_scene_desc: structure-of-arrays host
 *     buffers that mirror the crate's Scene / ShapeGroup / Shape / Path /
 *     Paint types (src/scene.rs:7-291, src/geometry.rs:78-104) with integer
 *     indices instead of nested Rust enums.
 *   - Matrices are the crate's Mat3 (src/math.rs:143-146): 9 floats,
 *     row-major, m[r][c] at index 3*r+c.
 *   - Colours are linear, non-premultiplied RGBA, as in Color (src/color.rs).
 *   - Entry points return dvg_status.  On error, dvg_last_error() gives a
 *     thread-local message; DVG_ERR_INVALID_SCENE carries the same reason
 *     strings as RenderError::InvalidScene (src/renderer/types.rs:83-88).
 *   - Calls on one context are serialised on that context's CUDA stream.
 *     A context may be used from one host thread at a time.
 *   - Scenes and batches belong to the context they were created on: destroy
 *     them before that context.
 */
#ifndef DVG_H
#define DVG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DVG_ABI_VERSION 2

typedef enum dvg_status {
    DVG_OK = 0,
    DVG_ERR_INVALID_SCENE = 1,    /* RenderError::InvalidScene */
    DVG_ERR_LAUNCH = 2,           /* RenderError::Launch (CUDA launch / runtime error) */
    DVG_ERR_DEVICE_LIMIT = 3,     /* a bounded device loop hit its cap; result not written */
    DVG_ERR_INVALID_ARGUMENT = 4, /* NULL pointer, bad enum, size mismatch in the call itself */
    DVG_ERR_OUT_OF_MEMORY = 5,
    DVG_ERR_NO_DEVICE = 6
} dvg_status;

/* Shape kinds: same ids as the crate's GPU constants (src/gpu/constants.rs:27-34). */
enum { DVG_SHAPE_CIRCLE = 0, DVG_SHAPE_RECT = 1, DVG_SHAPE_PATH = 2, DVG_SHAPE_ELLIPSE = 3 };
/* Paint kinds (src/gpu/constants.rs:36-43). */
enum { DVG_PAINT_NONE = 0, DVG_PAINT_SOLID = 1, DVG_PAINT_LINEAR = 2, DVG_PAINT_RADIAL = 3 };
/* FilterType (src/scene.rs:6-28); DVG_FILTER_GAUSSIAN is an addition of this library. */
enum { DVG_FILTER_BOX = 0, DVG_FILTER_TENT = 1, DVG_FILTER_RADIAL_PARABOLIC = 2, DVG_FILTER_HANN = 3,
       DVG_FILTER_GAUSSIAN = 4 };
/* FillRule (src/scene.rs:47-63). */
enum { DVG_FILL_NONZERO = 0, DVG_FILL_EVENODD = 1 };
/* StrokeJoin / StrokeCap (src/scene.rs:66-107).  The crate renders round joins and
 * caps only (the other values just widen bounds); this library also renders the
 * others for paths, in the forward pass and the interior adjoint (non-prefiltered):
 * bevel (the outer triangle at a vertex), miter (up to shape_miter_limit radii from
 * the vertex, else bevel), butt (the stroke ends at the end point's normal) and
 * square (one radius beyond the end).  Round (the default) is the crate's result
 * bit for bit.  Prefiltered coverage, the signed distance and the boundary sampling
 * of the edge term keep the crate's round geometry (the join and cap outline edges
 * are not sampled).  Other values are rejected as an invalid scene. */
enum { DVG_JOIN_MITER = 0, DVG_JOIN_BEVEL = 1, DVG_JOIN_ROUND = 2 };
enum { DVG_CAP_BUTT = 0, DVG_CAP_SQUARE = 1, DVG_CAP_ROUND = 2 };
/* Path flags. */
enum { DVG_PATH_CLOSED = 1u, DVG_PATH_DISTANCE_APPROX = 2u, DVG_PATH_HAS_THICKNESS = 4u };
/* Boundary-sampling random number generators. */
enum { DVG_RNG_PCG32 = 0, DVG_RNG_PHILOX = 1 };

/*
 * Scene description (host memory).  Replaces the Scene value passed by
 * reference to Renderer::render / render_backward (src/renderer/renderer.rs:39,548).
 *
 * shape_params per kind (Shape::geometry, src/scene.rs:151-180):
 *   CIRCLE  : center.x, center.y, radius, 0
 *   ELLIPSE : center.x, center.y, radius.x, radius.y
 *   RECT    : min.x, min.y, max.x, max.y
 *   PATH    : unused (geometry lives in the path_* arrays)
 * paint_params per kind (Paint, src/scene.rs:109-149):
 *   SOLID   : r, g, b, a
 *   LINEAR  : start.x, start.y, end.x, end.y      (+ stops)
 *   RADIAL  : center.x, center.y, radius.x, radius.y (+ stops)
 * Each group's fill and stroke must reference distinct paint entries: paint
 * gradients are returned per paint entry, which is how SceneGrad keeps one
 * DPaint per group fill / stroke (src/grad.rs:95-102).
 */
typedef struct dvg_scene_desc {
    uint32_t width, height;
    float background[4];            /* Scene::background */
    const float* background_image;  /* NULL, or width*height*4 floats (Scene::background_image) */
    uint32_t filter_type;           /* Scene::filter.filter_type */
    float filter_radius;            /* Scene::filter.radius */

    uint32_t num_shapes;
    const uint32_t* shape_kind;         /* [num_shapes] */
    const float* shape_params;          /* [num_shapes*4] */
    const float* shape_transform;       /* [num_shapes*9] Shape::transform */
    const float* shape_stroke_width;    /* [num_shapes] Shape::stroke_width (a radius, as in the crate) */
    const uint32_t* shape_stroke_join;  /* [num_shapes] or NULL (= round) */
    const uint32_t* shape_stroke_cap;   /* [num_shapes] or NULL (= round) */
    const float* shape_miter_limit;     /* [num_shapes] or NULL (= 4.0) */

    /* Paths (Path, src/geometry.rs:78-89).  Indexed per shape; ignored for other kinds. */
    const uint32_t* path_ctrl_offset;   /* [num_shapes] start in num_control_points */
    const uint32_t* path_ctrl_count;    /* [num_shapes] number of segments */
    const uint32_t* path_point_offset;  /* [num_shapes] start in points / thickness */
    const uint32_t* path_point_count;   /* [num_shapes] */
    const uint32_t* path_flags;         /* [num_shapes] DVG_PATH_* */
    const uint8_t* num_control_points;  /* flat: 0 line, 1 quadratic, 2 cubic */
    const float* points;                /* flat: 2 floats per point */
    const float* thickness;             /* flat: 1 float per point, or NULL if no path has thickness */
    uint32_t total_ctrl;                /* length of num_control_points */
    uint32_t total_points;              /* number of points (points has 2*total_points floats) */

    uint32_t num_groups;
    const uint32_t* group_shape_offset; /* [num_groups] start in group_shape_ids */
    const uint32_t* group_shape_count;  /* [num_groups] */
    const uint32_t* group_shape_ids;    /* flat ShapeGroup::shape_indices */
    uint32_t total_group_shapes;
    const uint32_t* group_fill_rule;    /* [num_groups] */
    const float* group_shape_to_canvas; /* [num_groups*9] */
    const float* group_canvas_to_shape; /* [num_groups*9] */
    const int32_t* group_fill_paint;    /* [num_groups] paint index or -1 */
    const int32_t* group_stroke_paint;  /* [num_groups] paint index or -1 */

    uint32_t num_paints;
    const uint32_t* paint_kind;         /* [num_paints] */
    const float* paint_params;          /* [num_paints*4] */
    const uint32_t* paint_stop_offset;  /* [num_paints] start in stop arrays */
    const uint32_t* paint_stop_count;   /* [num_paints] */
    const float* stop_offsets;          /* flat */
    const float* stop_colors;           /* flat RGBA */
    uint32_t total_stops;
} dvg_scene_desc;

/* RenderOptions (src/renderer/types.rs:10-39). Defaults: aa 1, path_tolerance 0.5,
 * 2x2 samples, seed 0, jitter 1, use_prefiltering 1. */
typedef struct dvg_render_options {
    float aa;
    float path_tolerance;
    uint32_t samples_x, samples_y;
    uint32_t seed;
    uint32_t jitter;
    uint32_t use_prefiltering;
} dvg_render_options;

/* BackwardOptions (src/backward/render.rs:19-32) plus the boundary-sampling knobs. */
typedef struct dvg_backward_options {
    uint32_t compute_translation;
    uint32_t boundary_samples;  /* 0 = width*height*spp, as the crate (src/renderer/backward_gpu.rs:396-398) */
    uint32_t rng;               /* DVG_RNG_PCG32 (the crate's generator) or DVG_RNG_PHILOX */
    uint32_t boundary_seed;     /* seed for the boundary pass; the crate uses RenderOptions::seed */
    uint32_t boundary_seed_from_options; /* 1: use RenderOptions::seed (crate behaviour) */
} dvg_backward_options;

/*
 * Gradient buffers (caller-owned, host or device memory depending on the call).
 * Flattened SceneGrad (src/grad.rs:113-126); every pointer may be NULL when the
 * caller does not want that part, except where noted.  Buffers are overwritten.
 */
typedef struct dvg_grads {
    float* d_shape_params;       /* [num_shapes*4] DShapeGeometry (circle/ellipse/rect) */
    float* d_shape_transform;    /* [num_shapes*9] DShape::transform */
    float* d_shape_stroke_width; /* [num_shapes]   DShape::stroke_width */
    float* d_points;             /* [total_points*2] DShapeGeometry::Path::points */
    float* d_thickness;          /* [total_points] DShapeGeometry::Path::thickness */
    float* d_group_transform;    /* [num_groups*9] DShapeGroup::shape_to_canvas */
    float* d_paint_params;       /* [num_paints*4] DPaint colour / start,end / center,radius */
    float* d_stop_offsets;       /* [total_stops] */
    float* d_stop_colors;        /* [total_stops*4] */
    float* d_filter_radius;      /* [1] DFilter::radius */
    float* d_background;         /* [4] SceneGrad::background */
    float* d_background_image;   /* [w*h*4] or NULL */
    float* d_translation;        /* [w*h*2] or NULL */
} dvg_grads;

typedef struct dvg_context dvg_context;
typedef struct dvg_scene dvg_scene;

/* Launch shape of the sample and boundary kernels (no counterpart in the crate; the
 * results do not depend on it beyond float summation order).
 * sample_layout: 1 = a warp holds all sub-samples of 32/spp neighbouring pixels
 *                (default), 0 = a warp holds one sub-sample of 32 pixels.
 * boundary_cell: boundary samples are sorted by cells of this many pixels square
 *                inside their 16x16 tile before evaluation: 2, 4 (default), 8 or 16.
 * fragment_slots: fragment codes kept per pixel sample by the forward pass of the
 *                fused calls (dvg_fwd_bwd_l2_device, batch steps) for the interior
 *                adjoint, which then skips its own hit tests for samples with at most
 *                this many fragments; 0 disables the cache, at most 64, default 16.
 *                Device memory: (2 * slots + 1) bytes per pixel sample of the scene
 *                (W * H * spp, rounded up to whole 16x16 tiles).
 * work_queue:    batches only: 0 = the forward and interior stages launch one CTA per
 *                work item (scene, tile, sub-sample), heaviest tiles first (default);
 *                1 = they launch as many persistent CTAs as the GPU holds at once, which
 *                take the items from a device counter in the same order.
 * forward_occupancy: the non-prefiltered forward kernel's register budget: 0 = 4 CTAs of
 *                256 threads per SM (64 registers, default), 1 = 3 CTAs (80 registers),
 *                2 = 2 CTAs (128 registers): fewer resident warps, fewer spills. */
typedef struct dvg_tuning {
    uint32_t sample_layout;
    uint32_t boundary_cell;
    uint32_t fragment_slots;
    uint32_t work_queue;
    uint32_t forward_occupancy;
} dvg_tuning;

/* Version of this ABI (DVG_ABI_VERSION). */
uint32_t dvg_abi_version(void);

/* Thread-local description of the last error on this thread. */
const char* dvg_last_error(void);

/* Replaces Renderer::new / Renderer::with_device (src/renderer/renderer.rs:25-36):
 * binds a CUDA device and creates the context's stream and scratch pool. */
dvg_status dvg_context_create(int device, dvg_context** out);
void dvg_context_destroy(dvg_context* ctx);
/* Retention of the last dvg_render for dvg_render_backward (see dvg_render); 1 by
 * default.  Turning it off releases the retained scene; with it off, dvg_render
 * writes no fragment codes and frees its scene at once. */
dvg_status dvg_context_set_retain(dvg_context* ctx, int enable);

/* Host preparation + upload.  Replaces prepare_scene / prepare_scene_backward and the
 * buffer uploads (src/renderer/prepare.rs:114, src/renderer/prepare_backward.rs:45,
 * src/renderer/renderer.rs:94-144).  The returned scene may be rendered many times. */
dvg_status dvg_scene_upload(dvg_context* ctx, const dvg_scene_desc* desc, dvg_scene** out);
void dvg_scene_destroy(dvg_scene* scene);

/* Renderer::render (src/renderer/renderer.rs:39-545) on an uploaded scene.
 * out_rgba: width*height*4 floats, un-premultiplied linear RGBA, row-major.
 * *_host variants take host pointers and block until the result is copied back;
 * *_device variants take device pointers, enqueue on the context stream and return. */
dvg_status dvg_render_host(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                           float* out_rgba);
dvg_status dvg_render_device(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                             float* out_rgba);

/* Renderer::render_backward (src/renderer/renderer.rs:548-564 ->
 * src/renderer/backward_gpu.rs:21-523) on an uploaded scene.
 * d_render: width*height*4 floats or NULL.  d_sdf: width*height floats or NULL, the
 * adjoint of dvg_render_sdf; as in the crate (src/backward/render.rs:171-188), every
 * sample of a pixel passes that pixel's full d_sdf to the closest-boundary adjoint
 * (it is not divided by the sample count). */
dvg_status dvg_render_backward_host(dvg_context* ctx, dvg_scene* scene,
                                    const dvg_render_options* opts,
                                    const dvg_backward_options* bopts,
                                    const float* d_render, const float* d_sdf, dvg_grads* grads);
dvg_status dvg_render_backward_device(dvg_context* ctx, dvg_scene* scene,
                                      const dvg_render_options* opts,
                                      const dvg_backward_options* bopts,
                                      const float* d_render, const float* d_sdf, dvg_grads* grads);

/* Signed distance field.  Replaces Renderer::render_sdf (src/renderer/renderer.rs:586-716,
 * src/gpu/kernels/sdf.rs:118-200): out = width*height floats, per pixel the mean over
 * its samples of the signed distance to the closest boundary of any group (searched
 * last group first), negative inside that group's fill; 0 without groups. */
dvg_status dvg_render_sdf_host(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts, float* out);
dvg_status dvg_render_sdf_device(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts, float* out);
dvg_status dvg_render_sdf(dvg_context* ctx, const dvg_scene_desc* desc, const dvg_render_options* opts, float* out);
/* Renderer::eval_positions (src/renderer/renderer.rs:719-848): the signed distance at
 * `count` canvas points (positions: 2*count floats, x then y). */
dvg_status dvg_eval_positions_host(dvg_context* ctx, dvg_scene* scene, const float* positions, uint64_t count,
                                   float* out);
dvg_status dvg_eval_positions_device(dvg_context* ctx, dvg_scene* scene, const float* positions, uint64_t count,
                                     float* out);
dvg_status dvg_eval_positions(dvg_context* ctx, const dvg_scene_desc* desc, const float* positions, uint64_t count,
                              float* out);
/* Renderer::eval_positions_backward -> render_backward_positions
 * (src/renderer/renderer.rs:567-583, src/backward/render.rs:213-281): gradients of
 * sum(d_values * sdf(positions)); points with d_value 0 are skipped; translation
 * gradients land on the pixel containing the point. */
dvg_status dvg_eval_positions_backward_host(dvg_context* ctx, dvg_scene* scene, const dvg_backward_options* bopts,
                                            const float* positions, uint64_t count, const float* d_values,
                                            dvg_grads* grads);
dvg_status dvg_eval_positions_backward_device(dvg_context* ctx, dvg_scene* scene, const dvg_backward_options* bopts,
                                              const float* positions, uint64_t count, const float* d_values,
                                              dvg_grads* grads);
dvg_status dvg_eval_positions_backward(dvg_context* ctx, const dvg_scene_desc* desc, const dvg_backward_options* bopts,
                                       const float* positions, uint64_t count, const float* d_values,
                                       dvg_grads* grads);

/* Render of an uploaded scene that allocates no device memory.  No counterpart in
 * the crate: it exists for callers that cannot call cudaMalloc while rendering (a
 * host application that fixes the device-memory budget up front, a plugin running
 * inside another framework's frame loop, code that must avoid the allocator's
 * implicit synchronisation).  Same inputs, output and result as dvg_render_device,
 * but the splat accumulators live in one file-scope device array of 5 MiB held by
 * every GPU that loads the library, so the canvas may have at most 512*512 pixels;
 * larger canvases return DVG_ERR_INVALID_ARGUMENT and launch nothing.  All calls on
 * a device share that array (each call clears it first); calls that overlap on the
 * GPU race on it.  The first call on a device looks up the array's address (with
 * the device current); make that first call before any stream capture begins.
 * The address is kept for the life of the process: after a cudaDeviceReset of
 * that device (which rebuilds its context and the array) do not call this entry
 * point again in the same process. */
dvg_status dvg_render_device_noalloc(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                     float* out_rgba);

/* One-shot forms mirroring the crate's call shape exactly: scene description in,
 * host image / host gradients out (upload, launch, read back).  With retention on
 * (the default, dvg_context_set_retain), dvg_render keeps its prepared scene, its
 * weight image and the per-sample fragment codes of its forward pass in the
 * context; a following dvg_render_backward whose description has the same bytes
 * (every scalar and array) and whose options are equal reuses them, as long as no
 * other call on the context rendered or drew weights in between.  Results are the
 * same either way (to float summation order). */
dvg_status dvg_render(dvg_context* ctx, const dvg_scene_desc* desc, const dvg_render_options* opts,
                      float* out_rgba);
dvg_status dvg_render_backward(dvg_context* ctx, const dvg_scene_desc* desc,
                               const dvg_render_options* opts, const dvg_backward_options* bopts,
                               const float* d_render, const float* d_sdf, dvg_grads* grads);

/* One scene split over several processes (each usually on its own GPU), for scenes
 * too slow for one device: each process renders a band of 16x16-pixel tiles and a
 * range of boundary samples, and the caller sums across processes between the calls
 * (for instance an NCCL all-reduce):
 *   dvg_shard_forward   -> sum accum_rgba and wsum over processes
 *   dvg_shard_resolve (+ dvg_l2_device, or any loss) on the whole image, every process
 *   dvg_shard_backward  -> sum the gradients over processes.
 * The sums equal a single-process render and backward up to float summation order.
 * tile_begin / tile_end index the scene's tiles in row-major order
 * (dvg_scene_tile_count); sample_begin / sample_end index the step's boundary
 * samples (bopts->boundary_samples, or W*H*spp when 0; clamped to that count).
 * No counterpart in the crate. */
typedef struct dvg_shard {
    uint32_t tile_begin, tile_end;
    uint64_t sample_begin, sample_end;
} dvg_shard;
dvg_status dvg_scene_tile_count(const dvg_scene* scene, uint32_t* tiles);
/* Number of groups binned to each tile (row-major; groups[n], n >= the tile count), the
 * per-tile work estimate for splitting the tiles by cost instead of by count.  Synchronises. */
dvg_status dvg_scene_tile_groups(const dvg_scene* scene, uint32_t* groups, uint32_t n);
/* Zeroes accum_rgba (W*H*4) and wsum (W*H) device buffers, then splats the samples of
 * the shard's tiles into them (pixels near the band's edges also receive the filter
 * splats of the neighbouring bands' samples: only the sums are complete).  With the
 * scene's fragment_slots > 0 it also keeps the samples' fragment codes for the
 * dvg_shard_backward of the same scene, options and tiles that follows. */
dvg_status dvg_shard_forward(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                             const dvg_shard* shard, float* accum_rgba, float* wsum);
/* The image from summed accumulators (weighted mean, un-premultiplied; the
 * background where no weight), W*H*4 device floats. */
dvg_status dvg_shard_resolve(dvg_context* ctx, dvg_scene* scene, const float* accum_rgba, const float* wsum,
                             float* out_rgba);
/* loss = sum((image - target)^2) into *loss (device float, may be NULL) and
 * d_render = 2 (image - target), n floats each, on device buffers. */
dvg_status dvg_l2_device(dvg_context* ctx, const float* image, const float* target, uint64_t n, float* d_render,
                         float* loss);
/* Zeroes the device gradient buffers, then adds the interior adjoint of the shard's
 * tiles and the edge-sampling term of its boundary samples; d_render (W*H*4) and
 * wsum (W*H) are the whole image's. */
dvg_status dvg_shard_backward(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                              const dvg_backward_options* bopts, const dvg_shard* shard, const float* d_render,
                              const float* wsum, dvg_grads* grads);

/* Forward + L2 loss + backward in one call on an uploaded scene (device pointers):
 * loss = sum((render - target)^2); d_render = 2*(render - target).
 * out_rgba (may be NULL), loss_out (device float, may be NULL).  No counterpart in
 * the crate: it fuses the render -> loss -> render_backward sequence a caller runs. */
dvg_status dvg_fwd_bwd_l2_device(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                 const dvg_backward_options* bopts, const float* target_rgba,
                                 float* out_rgba, float* loss_out, dvg_grads* grads);

/* Batches (no counterpart in the crate): many uploaded scenes stepped together.
 * A step renders every scene, forms the L2 loss against that scene's target, and
 * runs the backward pass — one kernel launch per stage for all scenes (work items
 * are (scene, tile, sub-sample) triples; boundary samples of all scenes are sorted
 * together by tile).  All scenes share opts / bopts.  The batch owns the images,
 * targets, gradients and scratch of every scene; dvg_batch_buffers returns device
 * pointers into them (write the targets there before stepping).
 * dvg_batch_step(use_graph=1) captures the step into a CUDA graph on its first call
 * and replays it afterwards; use_graph=0 enqueues the kernels directly. */
typedef struct dvg_batch dvg_batch;
dvg_status dvg_batch_create(dvg_context* ctx, dvg_scene* const* scenes, uint32_t count,
                            const dvg_render_options* opts, const dvg_backward_options* bopts,
                            dvg_batch** out);
void dvg_batch_destroy(dvg_batch* batch);
dvg_status dvg_batch_buffers(dvg_batch* batch, uint32_t index, float** image, float** target,
                             dvg_grads* grads);
dvg_status dvg_batch_step(dvg_batch* batch, int use_graph);
/* Copies the per-scene L2 losses of the last step to host memory (synchronises). */
dvg_status dvg_batch_losses(dvg_batch* batch, float* host_losses);

/* On-device optimisation step (no counterpart in the crate, whose callers update
 * parameters on the host and re-prepare the scene on every call).  Once set, every
 * dvg_batch_step also runs, after the backward pass: Adam (PyTorch's default form,
 * no weight decay) on the selected parameters of every scene, then rebuilds in
 * place every scene table derived from path points — segments, path and group
 * BVHs (the crate's median split, same leaf order), group canvas boxes, tile lists,
 * boundary-sampling lengths and CDFs — exactly as a fresh dvg_scene_upload of the
 * updated scene would build them.  The scenes' points / paint parameters are
 * updated in place.  Setting (or clearing, opts = NULL) resets the Adam moments and
 * step count and drops a captured graph (the next graph step recaptures).  Tile
 * lists of the batch's scenes are grown to their worst case (every group in every
 * tile); scenes for which that exceeds 2^28 entries return DVG_ERR_DEVICE_LIMIT. */
enum { DVG_OPT_POINTS = 1u, DVG_OPT_PAINTS = 2u };
typedef struct dvg_adam_options {
    float lr, beta1, beta2, eps;
    uint32_t params; /* DVG_OPT_POINTS | DVG_OPT_PAINTS */
} dvg_adam_options;
dvg_status dvg_batch_set_adam(dvg_batch* batch, const dvg_adam_options* opts);
/* Current path points (2*total_points floats) and paint parameters (4*num_paints)
 * of batch scene `index`, copied to host memory (either pointer may be NULL);
 * synchronises, and brings the scene's own handle up to date so it can be rendered
 * or differentiated outside the batch. */
dvg_status dvg_batch_scene_params(dvg_batch* batch, uint32_t index, float* host_points, float* host_paint_params);

/* Launch-shape tuning of an uploaded scene (see dvg_tuning).  dvg_scene_autotune times
 * dvg_fwd_bwd_l2_device on the scene with each warp layout, each boundary cell and each
 * fragment-cache size (device target image, width*height*4 floats; the scene's own
 * gradient buffers are used as scratch; a candidate's time is the median of three runs
 * after a warm one), keeps the fastest for later calls and returns it.  Synchronises. */
dvg_status dvg_scene_set_tuning(dvg_scene* scene, const dvg_tuning* tuning);
dvg_status dvg_scene_get_tuning(const dvg_scene* scene, dvg_tuning* tuning);
dvg_status dvg_scene_autotune(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                              const dvg_backward_options* bopts, const float* target_rgba, dvg_tuning* out);
/* The same for a batch: times directly enqueued steps (targets as set in the batch),
 * keeps the fastest and drops a captured graph so the next graph step recaptures. */
dvg_status dvg_batch_set_tuning(dvg_batch* batch, const dvg_tuning* tuning);
dvg_status dvg_batch_autotune(dvg_batch* batch, dvg_tuning* out);

/* 64-bit FNV-1a digest of an uploaded scene's prepared device tables (every table of
 * the scene arena, the tile offsets and the used tile entries, the boundary flag).
 * No counterpart in the crate: it lets a caller check that the on-device
 * re-preparation of an optimised scene built exactly the tables a fresh
 * dvg_scene_upload of the same parameters builds.  Synchronises. */
dvg_status dvg_scene_digest(dvg_context* ctx, dvg_scene* scene, uint64_t* digest);

/* Linear BVH (Morton codes, bitonic key sort, Karras topology, bottom-up bounds) over
 * `count` boxes (4 floats each: min x, min y, max x, max y), built on the GPU.  No
 * counterpart in the crate, whose BVHs are median splits built on the host (the
 * scene tables keep those: the crate's closest-point search breaks exact distance
 * ties by their traversal order).  A building block for callers that need a BVH over
 * many boxes built on the device; its tree equals a CPU build of the same steps.  Outputs (host memory, each may be NULL): keys_out[count] sorted keys
 * (Morton code << 32 | box index), children_out[2*(count-1)] (left, right) of the
 * internal nodes 0..count-2 (node ids >= count-1 are leaves count-1+k, k = sorted
 * position), bounds_out[4*(2*count-1)].  At most 2^24 boxes.  Synchronises. */
dvg_status dvg_lbvh_build(dvg_context* ctx, const float* boxes, uint32_t count, uint64_t* keys_out,
                          int32_t* children_out, float* bounds_out);

/* Number of kernels this library launched on the context since creation. */
uint64_t dvg_context_launch_count(const dvg_context* ctx);

/* The context's CUDA stream (a cudaStream_t) for callers that interleave their own work. */
void* dvg_context_stream(dvg_context* ctx);

/* Kernel timing (no counterpart in the crate, which has no tracing): when enabled,
 * every launcher call of this library on the context is bracketed by CUDA events on
 * the context stream.  dvg_context_profile synchronises, then fills up to cap entries
 * of (launcher name, total milliseconds, calls) accumulated since the last reset and
 * returns the number of distinct launchers.  Names are static strings. */
dvg_status dvg_context_set_profiling(dvg_context* ctx, int enable);
int dvg_context_profile(dvg_context* ctx, const char** names, double* total_ms, uint64_t* calls, int cap);
void dvg_context_profile_reset(dvg_context* ctx);

#ifdef __cplusplus
}
#endif
#endif /* DVG_H */
