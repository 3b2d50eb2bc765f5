// kernels.cuh — parameters and host launchers of the kernels in kernels.cu.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace dvgb {

// Per-thread fragment capacity of the interior adjoint (the crate's GPU kernel
// used 256, src/gpu/kernels/backward.rs:1657-1662).  Exceeding it sets
// ST_FRAGMENT_OVERFLOW and the call returns DVG_ERR_DEVICE_LIMIT.
constexpr int MAX_FRAGMENTS = 96;
// Filter radii up to this (ceil) use the shared-memory tile+halo splat.
constexpr int MAX_SMEM_RI = 8;
// Boundary samples are counting-sorted by cell x cell-pixel cells of their tile
// (cell in {2, 4, 8, 16}) and, inside a cell, by class (fill or stroke, path or other
// shape: the code they run); bnd_buckets(cell) buckets per tile; scratch counts hold
// 2 * tiles * BND_MAX_BUCKETS + 1.
constexpr int BND_CLASSES = 4;
constexpr int BND_MAX_BUCKETS = (16 / 2) * (16 / 2) * BND_CLASSES;
inline int bnd_buckets(int cell) { return (16 / cell) * (16 / cell) * BND_CLASSES; }
// Ints of boundary-sort scratch for `tiles` tiles: counts, offsets (+1) and the
// two-level scan's chunk totals, bases and grand total.
inline size_t bnd_count_ints(size_t tiles) {
    const size_t b = tiles * BND_MAX_BUCKETS;
    return 2 * b + 1 + 2 * ((b + 4095) / 4096) + 1;
}

// Fragment cache of the fused forward -> interior paths: the forward stores, per
// pixel sample, the codes (2 * tile-list entry + 0 stroke / 1 fill) of the fragments
// it composited, and the interior adjoint reads them back instead of repeating the
// hit tests.  Codes are 16-bit (tile lists up to FRAG_MAX_ENTRIES entries), stored
// slot-major (slot k of sample s at k * samples + s, samples = tiles * spp * 256) so
// a warp's lanes touch consecutive halves; a count of FRAG_NONE marks a sample the
// interior re-tests (more fragments than slots, a longer tile list, or a sample
// point that the interior's normalise-and-rescale does not reproduce exactly).
// Share of a styled stroke's edge samples drawn on its join and cap edges.
constexpr float JOIN_CAP_SHARE = 0.25f;
constexpr int FRAG_MAX_ENTRIES = 32767;
constexpr uint8_t FRAG_NONE = 0xff;
constexpr int FRAG_MAX_SLOTS = 64;

struct SampleParams {
    int sxn, syn;
    uint32_t seed;
    bool jitter;
    int layout;  // 1: a warp holds all sub-samples of 32/spp pixels; 0: one sub-sample of 32 pixels
    uint16_t* frag;  // fragment codes (NULL: no cache)
    uint8_t* frag_n; // per-sample code count or FRAG_NONE
    int frag_slots;  // codes kept per sample (<= FRAG_MAX_SLOTS)
    int tile_base, tile_count;  // the tiles a single-scene launch covers (count 0: all)
    int fwd_occ;  // dvg_tuning.forward_occupancy: k_forward at 4 - fwd_occ CTAs per SM
};
// Work items of a batched stage (work[i] = (scene, tile + tiles * sub-sample round),
// heaviest first).  counter == nullptr: one CTA per item, item = blockIdx.x.  Otherwise
// the CTAs are persistent (as many as the GPU holds at once) and take the next item from
// *counter until the list is done; the counter is zeroed before the launch.  Every CTA
// makes at most items / gridDim.x + 2 atomic increments, so the loop always ends.
#ifdef __CUDACC__
template <typename F>
__device__ __forceinline__ void for_each_item(int items, int* counter, F&& body) {
    if (!counter) {
        if ((int)blockIdx.x < items) body((int)blockIdx.x);
        return;
    }
    __shared__ int s_item;
    for (;;) {
        __syncthreads();  // the previous item is done with shared memory and s_item
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int i = s_item;
        if (i >= items) return;
        body(i);
    }
}
#endif
// Grid width of a single-scene sample launch: the tiles it covers.
inline int launch_tiles(const DevScene& S, const SampleParams& sp) {
    return sp.tile_count > 0 ? sp.tile_count : S.tiles_x * S.tiles_y;
}
// Bytes of a fragment cache with `slots` codes per sample for one scene.
inline size_t frag_cache_bytes(int tiles, int spp, int slots) {
    const size_t samples = (size_t)tiles * spp * 256;
    return samples * (2 * (size_t)slots + 1);
}
struct BoundaryParams {
    uint64_t num_samples;  // one past the last sample index of this launch
    uint64_t sample_base;  // first sample index of this launch
    uint64_t slot_base;    // sample index stored in scratch slot 0
    uint32_t seed;
    int rng;   // 0 PCG32, 1 Philox
    int cell;  // boundary sort cell edge in pixels (2, 4, 8 or 16)
    // the step's boundary samples / (W*H*spp): the crate draws W*H*spp samples and its
    // edge term carries no 1/N, so another count rescales each sample's pdf (1: exact)
    float pdf_scale;
};
// One drawn edge sample (64 bytes), kept in scratch between the boundary stages.
struct BSample {
    float bx, by;  // boundary point, normalised canvas units
    float nx, ny;  // canvas-space normal
    float lx, ly;  // shape-space boundary point
    float pdf, t;  // combined pdf, raw random t
    int shape, group, pixel;
    int base_point_id, point_id;
    float bt;
    int is_stroke, scene;  // scene: index in a batch (0 for single-scene calls)
};
// One scene of a batch: its tables, options, gradient pointers, per-scene
// output buffers and its ranges in the batch-wide work numbering.
struct BatchEntry {
    DevScene S;
    SampleParams sp;
    GradPtrs G;
    float* accum;
    float* wsum;
    float* image;
    const float* target;
    float* d_render;
    float* loss;
    int item_off;    // first (tile, sub-sample) work item
    int tile_off;    // first tile in the batch-wide tile numbering
    uint64_t b_off;  // first boundary sample in the batch-wide numbering
    uint64_t nb;     // boundary samples of this scene
    uint32_t bseed;
    int rng;
    float bscale;  // nb / (W*H*spp), as BoundaryParams::pdf_scale
};

// Per-scene state of the on-device optimisation step (Adam + scene re-preparation).
struct RefitEntry {
    float* m_points;  // Adam first / second moments, 2 per point
    float* v_points;
    float* m_paints;  // 4 per paint (NULL when paints are not optimised)
    float* v_paints;
    int* sort_ids;     // scratch: 2 * sort_n ints
    float* sort_keys;  // scratch: 2 * sort_n floats
    int sort_n;        // max(total segments, total group shape entries)
    int n_points, n_paints;
    float4* g_bbox;    // the scene's canvas-space group boxes (tile binning input)
};
struct AdamParams {
    float lr, beta1, beta2, eps;
    int points, paints;  // which parameter sets are stepped
};

// Device buffers of one linear BVH over n boxes (lbvh.cu): keys[lbvh_padded(n)],
// children[n-1], parent[2n-1], flags[n-1], bounds[2n-1], leaf_item[n], extent[1].
struct LbvhBufs {
    uint64_t* keys;
    int2* children;
    int* parent;
    int* flags;
    float4* bounds;
    int* leaf_item;
    float4* extent;
};
int lbvh_padded(int n);

// Launchers (all asynchronous on `stream`).  Each returns the number of kernels launched.
int launch_binning(const DevScene& S, const float4* g_bbox, int* counts, int* offsets, int* entries_or_null,
                   cudaStream_t stream);
int launch_forward(const DevScene& S, const SampleParams& sp, float* accum, float* wsum, unsigned* status,
                   cudaStream_t stream);
int launch_forward_prefilter(const DevScene& S, const SampleParams& sp, float* accum, float* wsum, unsigned* status,
                             cudaStream_t stream);
int launch_weights(const DevScene& S, const SampleParams& sp, float* wsum, cudaStream_t stream);
int launch_resolve(const DevScene& S, const float* accum, const float* wsum, float* out, cudaStream_t stream);
int launch_interior(const DevScene& S, const SampleParams& sp, const float* d_render, const float* wsum,
                    const GradPtrs& G, unsigned* status, cudaStream_t stream);
int launch_interior_prefilter(const DevScene& S, const SampleParams& sp, const float* d_render, const float* wsum,
                              const GradPtrs& G, unsigned* status, cudaStream_t stream);
// Boundary pass in chunks of at most `capacity` samples; scratch: samples[capacity],
// key[capacity], order[capacity], counts[2*tiles*BND_MAX_BUCKETS+1].
int launch_boundary(const DevScene& S, const BoundaryParams& bp, const float* d_render, const float* wsum,
                    const GradPtrs& G, BSample* samples, int* key, int* counts, int* order, uint64_t capacity,
                    cudaStream_t stream);
int launch_finalize_background(const DevScene& S, const GradPtrs& G, cudaStream_t stream);
int launch_fill_background(const DevScene& S, float* out, cudaStream_t stream);
// Batched launchers: B (device) holds one BatchEntry per scene; work[i] = (scene, tile +
// tiles * sub-sample round) is the i-th work item, in any order (the batch lists the
// heaviest tiles first).  counter(s): null for one CTA per item, else zeroed device ints
// for persistent CTAs (see for_each_item; launch_interior_batch takes two, one per
// kernel).  which: 0 resolve, 1 L2, 2 background.
int launch_forward_batch(const BatchEntry* B, const int2* work, int items, int* counter, int max_ri, int occ,
                         cudaStream_t stream);
int launch_forward_prefilter_batch(const BatchEntry* B, const int2* work, int items, int* counter, int max_ri,
                                   unsigned* status, cudaStream_t stream);
int launch_pixels_batch(const BatchEntry* B, int nscenes, size_t max_pixels, int which, cudaStream_t stream);
int launch_interior_batch(const BatchEntry* B, const int2* work, int items, int* counters, unsigned* status,
                          cudaStream_t stream);
int launch_interior_prefilter_batch(const BatchEntry* B, const int2* work, int items, int* counter, unsigned* status,
                                    cudaStream_t stream);
int launch_boundary_batch(const BatchEntry* B, int nscenes, uint64_t total, int total_tiles, int cell, bool styled,
                          BSample* samples, int* key, int* counts, int* order, cudaStream_t stream);
// Optimisation step: Adam on the selected parameters of every scene, then the
// scene tables that depend on path points are rebuilt in place (segments, path and
// group BVHs, group canvas boxes, boundary-sampling tables).  Tile binning is
// re-run per scene by the caller afterwards.
int launch_adam_batch(BatchEntry* B, const RefitEntry* R, int nscenes, int max_params, const AdamParams& ap,
                      int* step, cudaStream_t stream);
int launch_refit_batch(BatchEntry* B, const RefitEntry* R, int nscenes, int max_paths, int max_groups,
                       unsigned* status, cudaStream_t stream);
// Signed distance field: per-pixel mean over samples, per-point values, and the
// adjoints of both (d_sdf image / per-point d_values) into G.
int launch_render_sdf(const DevScene& S, const SampleParams& sp, float* out, unsigned* status, cudaStream_t stream);
int launch_eval_positions(const DevScene& S, const float2* pos, uint64_t n, float* out, unsigned* status,
                          cudaStream_t stream);
int launch_sdf_backward(const DevScene& S, const SampleParams& sp, const float* d_sdf, const GradPtrs& G,
                        bool translation, unsigned* status, cudaStream_t stream);
int launch_positions_backward(const DevScene& S, const float2* pos, uint64_t n, const float* d_values,
                              const GradPtrs& G, bool translation, unsigned* status, cudaStream_t stream);
// Linear BVH over n boxes into L (leaf_item[k] = item_map[box index], or the box
// index without a map).
int launch_lbvh_build(const float4* boxes, int n, const int* item_map, LbvhBufs& L, cudaStream_t stream);
int launch_l2(const float* img, const float* target, size_t n, float* d_render, float* loss, cudaStream_t stream);

}  // namespace dvgb
