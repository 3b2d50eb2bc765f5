// kernels.cu — sm_100a kernels of the render / backward hot path.
//
//   k_bin_count / k_bin_scan / k_bin_write  tile binning of groups (group order kept)
//   k_forward      per (tile, sub-sample) CTA: scene evaluation + filtered splat
//                  into a shared-memory tile+halo accumulator, flushed once
//   k_weights      filter-weight image only (backward without a preceding forward)
//   k_resolve      Σ(c·w)/Σw and un-premultiply            (forward.rs:294-334)
//   k_interior     interior adjoint per sample             (backward/render.rs:95-169)
//   k_interior_cached  the same for samples whose fragments the forward cached
//   k_boundary     edge sampling adjoint per boundary sample (backward/boundary.rs:141-196)
//   k_l2           L2 loss and d_render
//
// Built with -fmad=false (see device.cuh).
#include <algorithm>

#include "device.cuh"
#include "kernels.cuh"

// Minimum resident CTAs per SM for the scene-evaluation kernels (register cap =
// 65536 / (threads * value)); chosen by measurement on B200.
// (the non-prefiltered forward is compiled for 2, 3 and 4, see dvg_tuning.forward_occupancy)
#ifndef DVG_MINB_INT
#define DVG_MINB_INT 2
#endif
#ifndef DVG_MINB_BND
#define DVG_MINB_BND 16  // 32 registers: more warps for the two-lane edge evaluation outweigh its spills
#endif
#ifndef DVG_MINB_LEAN
#define DVG_MINB_LEAN 4
#endif

namespace dvgb {

// ------------------------------------------------------------------ tile binning
// One CTA per tile scans all group boxes; the crate bins on the GPU and sorts on
// the host (src/renderer/renderer.rs:254-384); scanning in group order keeps the
// compositing order without a sort.  Edge tiles extend to infinity so that any
// point clamped to an edge tile is covered.
__device__ __forceinline__ bool tile_hits(const DevScene& S, int tile, float4 b) {
    int tx = tile % S.tiles_x, ty = tile / S.tiles_x;
    float x0 = tx == 0 ? -INFINITY : (float)(tx * TILE);
    float y0 = ty == 0 ? -INFINITY : (float)(ty * TILE);
    float x1 = tx == S.tiles_x - 1 ? INFINITY : (float)((tx + 1) * TILE);
    float y1 = ty == S.tiles_y - 1 ? INFINITY : (float)((ty + 1) * TILE);
    return !(b.z < x0 || b.x > x1 || b.w < y0 || b.y > y1);
}
__global__ void __launch_bounds__(256) k_bin_count(DevScene S, const float4* g_bbox, int* counts) {
    int tile = blockIdx.x;
    int total = 0;
    for (int base = 0; base < S.num_groups; base += blockDim.x) {
        int g = base + threadIdx.x;
        bool hit = false;
        if (g < S.num_groups) {
            int4 gi = S.g_info[g];
            hit = (gi.x >= 0 || gi.y >= 0) && tile_hits(S, tile, g_bbox[g]);
        }
        total += __syncthreads_count(hit);
    }
    if (threadIdx.x == 0) counts[tile] = total;
}
// Exclusive scan of tile counts (single CTA of 1024 threads, any length).
__global__ void __launch_bounds__(1024) k_bin_scan(const int* counts, int n, int* offsets) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < n; base += 1024) {
        int i = base + threadIdx.x;
        int v = i < n ? counts[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int w = warp_sums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        int excl = carry + (wid > 0 ? warp_sums[wid - 1] : 0) + x - v;
        if (i < n) offsets[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) offsets[n] = carry;
}
// Two-level exclusive scan for long count arrays (the boundary sort's buckets): each
// CTA scans 4096 counts and leaves its total in part[], one CTA scans the totals, a
// third pass adds each CTA's base.  offsets[n] receives the grand total.
constexpr int SCAN_CHUNK = 4096;
__global__ void __launch_bounds__(1024) k_scan_chunks(const int* counts, int n, int* offsets, int* part) {
    __shared__ int warp_sums[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int base = blockIdx.x * SCAN_CHUNK + 4 * threadIdx.x;
    int v[4], t = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = base + k < n ? counts[base + k] : 0;
        t += v[k];
    }
    int x = t;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = warp_sums[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    int excl = (wid > 0 ? warp_sums[wid - 1] : 0) + x - t;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (base + k < n) offsets[base + k] = excl;
        excl += v[k];
    }
    if (threadIdx.x == 1023) part[blockIdx.x] = warp_sums[31];
}
__global__ void __launch_bounds__(1024) k_scan_add(int* offsets, int n, const int* part_offsets) {
    const int i = blockIdx.x * SCAN_CHUNK + 4 * threadIdx.x;
    const int add = part_offsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (i + k < n) offsets[i + k] += add;
}
// Exclusive scan of counts[n] into offsets[n + 1]; part: scratch of scan_part_ints(n) ints.
inline int scan_chunks(int n) { return (n + SCAN_CHUNK - 1) / SCAN_CHUNK; }
int launch_scan(const int* counts, int n, int* offsets, int* part, cudaStream_t stream) {
    const int c = scan_chunks(n);
    if (c <= 1) {
        k_bin_scan<<<1, 1024, 0, stream>>>(counts, n, offsets);
        return 1;
    }
    k_scan_chunks<<<c, 1024, 0, stream>>>(counts, n, offsets, part);
    k_bin_scan<<<1, 1024, 0, stream>>>(part, c, part + c);  // part + c: the chunks' bases, then the total
    k_scan_add<<<c, 1024, 0, stream>>>(offsets, n, part + c);
    cudaMemcpyAsync(offsets + n, part + 2 * c, sizeof(int), cudaMemcpyDeviceToDevice, stream);
    return 3;
}

__global__ void __launch_bounds__(256) k_bin_write(DevScene S, const float4* g_bbox, const int* offsets,
                                                   int* entries) {
    __shared__ int warp_counts[8];
    int tile = blockIdx.x;
    int cursor = offsets[tile];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < S.num_groups; base += blockDim.x) {
        int g = base + threadIdx.x;
        bool hit = false;
        if (g < S.num_groups) {
            int4 gi = S.g_info[g];
            hit = (gi.x >= 0 || gi.y >= 0) && tile_hits(S, tile, g_bbox[g]);
        }
        unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) warp_counts[wid] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < 8; ++w) {
            if (w < wid) before += warp_counts[w];
            total += warp_counts[w];
        }
        if (hit) entries[cursor + before + __popc(m & ((1u << lane) - 1u))] = g;
        cursor += total;
        __syncthreads();
    }
}

// ------------------------------------------------------------------ forward
// One CTA = one 16x16 tile at one sub-sample (sx, sy); thread = pixel.  Every
// thread of the CTA walks the same group list, so group data loads are uniform.
__device__ __forceinline__ void forward_body(const DevScene& S, const SampleParams& sp, int tile, int round,
                                             float* accum, float* wsum, float* sm) {
    const int ri = S.filter_ri;
    const int HW = TILE + 2 * ri;
    const bool use_sm = ri <= MAX_SMEM_RI;
    const int tx = tile % S.tiles_x, ty = tile / S.tiles_x;
    const int spp = sp.sxn * sp.syn;
    const int s_in_tile = round * 256 + (int)threadIdx.x;
    const int pix = sp.layout ? s_in_tile / spp : (int)threadIdx.x, sub = sp.layout ? s_in_tile % spp : round;
    const int x = tx * TILE + (pix % TILE), y = ty * TILE + (pix / TILE);
    if (use_sm)
        for (int i = threadIdx.x; i < HW * HW * 5; i += blockDim.x) sm[i] = 0.0f;
    __syncthreads();
    const int off = S.tile_offsets[tile];
    const int n = S.tile_offsets[tile + 1] - off;
    const int* list = S.tile_entries + off;
    if (x < S.width && y < S.height) {
        const int sx = sub % sp.sxn, sy = sub / sp.sxn;
        const float2 pt = sample_pos(x, y, sx, sy, sp.sxn, sp.syn, S.width, sp.seed, sp.jitter);
        // Fragment cache (see SampleParams): kept only where the interior pass, which
        // normalises the sample point by the canvas size and scales it back
        // (src/backward/render.rs:111, src/backward/sampling.rs:91), tests the same point.
        const size_t fstride = (size_t)S.tiles_x * S.tiles_y * spp * 256;
        const size_t sid = ((size_t)tile * spp + round) * 256 + threadIdx.x;
        const bool cache = sp.frag != nullptr && n <= FRAG_MAX_ENTRIES &&
                           (pt.x / (float)S.width) * (float)S.width == pt.x &&
                           (pt.y / (float)S.height) * (float)S.height == pt.y;
        int nf = 0;
        float4 acc = background_premul(S, y * S.width + x);
        for (int e = 0; e < n; ++e) {
            const int g = __ldg(&list[e]);
            // stroke first, then fill; one paint call site for both
            const int4 gi = __ldg(&S.g_info[g]);
            const float2 lp = xf9(S.g_c2s + 9 * g, pt);
            int hitp[2];
            hitp[0] = gi.y >= 0 && group_within(S, g, lp) ? gi.y : -1;
            hitp[1] = gi.x >= 0 && group_inside(S, g, lp, gi.z) ? gi.x : -1;
#pragma unroll 1
            for (int which = 0; which < 2; ++which)
                if (hitp[which] >= 0) {
                    over(acc, paint_color(S, hitp[which], pt));
                    if (cache) {
                        if (nf < sp.frag_slots) sp.frag[(size_t)nf * fstride + sid] = (uint16_t)(2 * e + which);
                        ++nf;
                    }
                }
        }
        if (sp.frag) sp.frag_n[sid] = cache && nf <= sp.frag_slots ? (uint8_t)nf : FRAG_NONE;
        splat_sample(S, x, y, tx, ty, ri, HW, use_sm, pt, acc, sm, accum, wsum);
    }
    if (!use_sm) return;
    __syncthreads();
    flush_splat(S, tx, ty, ri, HW, sm, accum, wsum);
}
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_forward(DevScene S, SampleParams sp, float* accum, float* wsum,
                                                       unsigned* status) {
    extern __shared__ float sm[];
    (void)status;
    forward_body(S, sp, sp.tile_base + blockIdx.x, blockIdx.y, accum, wsum, sm);
}
// Batched forward: one flat grid over every (scene, tile, sub-sample) work item.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_forward_batch(const BatchEntry* __restrict__ B,
                                                             const int2* __restrict__ work, int items, int* counter) {
    extern __shared__ float sm[];
    for_each_item(items, counter, [&](int i) {
        const int2 wk = work[i];  // (scene, tile + tiles * sub-sample round)
        const BatchEntry& E = B[wk.x];
        const int tiles = E.S.tiles_x * E.S.tiles_y;
        forward_body(E.S, E.sp, wk.y % tiles, wk.y / tiles, E.accum, E.wsum, sm);
    });
}

// Weight image only (rasterize_weights_f32, forward.rs:1505-1564).
__global__ void __launch_bounds__(256) k_weights(DevScene S, SampleParams sp, float* wsum) {
    const int tile = sp.tile_base + blockIdx.x, sub = blockIdx.y;
    const int tx = tile % S.tiles_x, ty = tile / S.tiles_x;
    const int x = tx * TILE + (threadIdx.x % TILE), y = ty * TILE + (threadIdx.x / TILE);
    if (x >= S.width || y >= S.height) return;
    const int ri = S.filter_ri;
    const int sx = sub % sp.sxn, sy = sub / sp.sxn;
    const float2 pt = sample_pos(x, y, sx, sy, sp.sxn, sp.syn, S.width, sp.seed, sp.jitter);
    for (int dy = -ri; dy <= ri; ++dy)
        for (int dx = -ri; dx <= ri; ++dx) {
            int xx = x + dx, yy = y + dy;
            if (xx < 0 || yy < 0 || xx >= S.width || yy >= S.height) continue;
            float w = filter_weight(S.filter_type, S.filter_radius, (float)xx + 0.5f - pt.x, (float)yy + 0.5f - pt.y);
            if (w > 0.0f) atomicAdd(wsum + (size_t)yy * S.width + xx, w);
        }
}

__global__ void k_resolve(DevScene S, const float* accum, const float* wsum, float* out) {
    size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)S.width * S.height) return;
    float r = S.bg[0], g = S.bg[1], b = S.bg[2], a = S.bg[3];
    float w = wsum[p];
    if (w > 0.0f) {
        float4 c = reinterpret_cast<const float4*>(accum)[p];
        r = c.x / w;
        g = c.y / w;
        b = c.z / w;
        a = c.w / w;
    }
    if (a > 1.0e-8f) {
        r = r / a;
        g = g / a;
        b = b / a;
    }
    reinterpret_cast<float4*>(out)[p] = make_float4(r, g, b, a);
}

// ------------------------------------------------------------------ backward helpers
// ------------------------------------------------------------------ interior backward
// Per sample: gather d_color (filters.rs:70-103), recompute the fragments of
// sample_color (sampling.rs:76-224) and back-propagate through compositing,
// paints, background and the filter (filters.rs:106-156).  The fragment list comes
// from the forward's fragment cache or is rebuilt from the BVHs; only (fragment
// code, transmittance) pairs live in per-thread local memory.  The adjoint loop
// walks the tile's group list in the same order on every lane so solid-paint
// gradients reduce across the warp before one atomic.
//
// LEAN: the kernel takes only the samples with cached fragments and carries no hit
// tests (fewer registers, more resident warps for its load chains); otherwise it
// takes every sample without a cache entry (all samples when there is no cache).
// Each sample is handled by exactly one of the two launches.
template <bool LEAN>
__device__ __forceinline__ void interior_body(const DevScene& S, const SampleParams& sp, int tile, int round,
                                              const float* d_render, const float* wsum, const GradPtrs& G,
                                              unsigned* status) {
    __shared__ float red[8][6];
    const int tx = tile % S.tiles_x, ty = tile / S.tiles_x;
    const int spp = sp.sxn * sp.syn;
    const int s_in_tile = round * 256 + (int)threadIdx.x;
    const int pix = sp.layout ? s_in_tile / spp : (int)threadIdx.x, sub = sp.layout ? s_in_tile % spp : round;
    const int x = tx * TILE + (pix % TILE), y = ty * TILE + (pix / TILE);
    const size_t fstride = (size_t)S.tiles_x * S.tiles_y * spp * 256;
    const size_t sid = ((size_t)tile * spp + round) * 256 + threadIdx.x;
    const bool inside = x < S.width && y < S.height;
    const int cn = inside && sp.frag ? (int)__ldcs(&sp.frag_n[sid]) : (int)FRAG_NONE;
    const bool valid = inside && (LEAN ? cn != (int)FRAG_NONE : cn == (int)FRAG_NONE);
    if (!__syncthreads_or(valid)) return;  // uniform per CTA
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int off = S.tile_offsets[tile];
    const int n = S.tile_offsets[tile + 1] - off;
    const int* list = S.tile_entries + off;
    const int W = S.width, H = S.height;

    float2 ps = make_float2(0.0f, 0.0f), pt = make_float2(0.0f, 0.0f);
    int pixel = 0;
    float4 dcol = make_float4(0, 0, 0, 0), bg = make_float4(0, 0, 0, 0);
    if (valid) {
        const int sx = sub % sp.sxn, sy = sub / sp.sxn;
        ps = sample_pos(x, y, sx, sy, sp.sxn, sp.syn, W, sp.seed, sp.jitter);
        float2 npt = make_float2(ps.x / (float)W, ps.y / (float)H);  // render.rs:111
        pt = make_float2(npt.x * (float)W, npt.y * (float)H);       // sampling.rs:91
        pixel = y * W + x;
        bg = background_premul(S, pixel);
        dcol = gather_d_color(S, d_render, wsum, ps);
    }
    // Pass 1: fragments in order (stroke before fill within a group).
    int code[MAX_FRAGMENTS];
    float tr[MAX_FRAGMENTS];
    int nf = 0;
    bool overflow = false;
    float4 acc = bg;
    if (valid) {
        // Either the forward's cached fragment codes (one fragment per step) or the
        // tile's group list with both hit tests (up to two fragments per step).
        const int steps = LEAN ? cn : n;
        for (int k = 0; k < steps; ++k) {
            int e, hitp[2];
            if constexpr (LEAN) {
                const int c0 = __ldcs(&sp.frag[(size_t)k * fstride + sid]);
                e = c0 >> 1;
                const int4 gi = __ldg(&S.g_info[__ldg(&list[e])]);
                hitp[0] = (c0 & 1) ? -1 : gi.y;
                hitp[1] = (c0 & 1) ? gi.x : -1;
            } else {
                e = k;
                const int g = __ldg(&list[e]);
                const int4 gi = __ldg(&S.g_info[g]);
                const float2 lp = xf9(S.g_c2s + 9 * g, pt);
                hitp[0] = gi.y >= 0 && group_within(S, g, lp) ? gi.y : -1;
                hitp[1] = gi.x >= 0 && group_inside(S, g, lp, gi.z) ? gi.x : -1;
            }
#pragma unroll 1
            for (int which = 0; which < 2; ++which) {
                if (hitp[which] < 0) continue;
                float4 c = paint_color(S, hitp[which], pt);
                over(acc, c);
                if (nf < MAX_FRAGMENTS) {
                    code[nf] = 2 * e + which;
                    tr[nf] = c.w;
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
    // Final colour and the adjoint at the end of compositing (sampling.rs:161-174).
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
        // Pass 2: transmittance after each fragment, T_i = prod_{j>i}(1 - a_j).
        float run = 1.0f;
        for (int i = nf - 1; i >= 0; --i) {
            float a = tr[i];
            tr[i] = run;
            run = run * (1.0f - a);
        }
        // background adjoint after all fragments
        float4 dbg = make_float4(dcr * run, dcg * run, dcb * run, dca * run);
        if (S.bg_image) {
            float* b = G.d_background_image;
            if (b) {
                add_if(b + 4 * (size_t)pixel + 0, dbg.x);
                add_if(b + 4 * (size_t)pixel + 1, dbg.y);
                add_if(b + 4 * (size_t)pixel + 2, dbg.z);
                add_if(b + 4 * (size_t)pixel + 3, dbg.w);
            }
            dbg = make_float4(0, 0, 0, 0);
        }
        dcol = dbg;  // reused below as this sample's constant-background adjoint
    } else if (active) {
        // no fragment: accumulate_background_grad(d_color) (sampling.rs:121-127)
        if (S.bg_image) {
            float* b = G.d_background_image;
            if (b) {
                add_if(b + 4 * (size_t)pixel + 0, dcol.x);
                add_if(b + 4 * (size_t)pixel + 1, dcol.y);
                add_if(b + 4 * (size_t)pixel + 2, dcol.z);
                add_if(b + 4 * (size_t)pixel + 3, dcol.w);
            }
            dcol = make_float4(0, 0, 0, 0);
        }
    }
    if (!active) dcol = make_float4(0, 0, 0, 0);

    // Pass 3: forward over the fragments with the compositing adjoint (sampling.rs:175-210).
    // The warp visits only the (group, stroke/fill) entries some lane hit: each round
    // takes the smallest next fragment code over the warp, so lanes stay in step for
    // the warp-reduced solid-paint gradients while entries nobody hit cost nothing.
    int cur = 0;
    float4 prev = bg;
    while (true) {
        const int mine = cur < nf ? code[cur] : 0x7fffffff;
        const int nxt = __reduce_min_sync(0xffffffffu, mine);
        if (nxt == 0x7fffffff) break;
        const int e = nxt >> 1, which = nxt & 1;  // code = 2 * entry + (0 stroke, 1 fill)
        const int g = __ldg(&list[e]);
        const int4 gi = __ldg(&S.g_info[g]);
        const int p = which == 0 ? gi.y : gi.x;
        const bool has = mine == nxt;
        float4 dv = make_float4(0, 0, 0, 0);
        if (has) {
            const float4 c = paint_color(S, p, pt);
            float T = tr[cur];
            float r_ = dcr * T, g_ = dcg * T, b_ = dcb * T, a_ = dca * T;
            float d_alpha = a_ * (1.0f - prev.w);
            d_alpha += r_ * (c.x - prev.x) + g_ * (c.y - prev.y) + b_ * (c.z - prev.z);
            dv = make_float4(r_ * c.w, g_ * c.w, b_ * c.w, d_alpha);
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
        } else {
            float2 dtr = make_float2(0.0f, 0.0f);
            d_gradient_paint_warp(S, G, p, pt, dv, has, &dtr);
            if (has && G.d_translation) {
                add_if(G.d_translation + 2 * (size_t)pixel, dtr.x);
                add_if(G.d_translation + 2 * (size_t)pixel + 1, dtr.y);
            }
        }
    }
    // Filter-radius adjoint (filters.rs:106-156) and the constant-background adjoint.
    const float dradius = active ? filter_radius_adjoint(S, d_render, wsum, ps, ret) : 0.0f;
    float v[5] = {dcol.x, dcol.y, dcol.z, dcol.w, dradius};
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
        for (int k = 0; k < 5; ++k) red[wid][k] = v[k];
    __syncthreads();
    if (threadIdx.x < 5) {
        float s = 0.0f;
        for (int w = 0; w < 8; ++w) s += red[w][threadIdx.x];
        if (threadIdx.x < 4)
            add_if(G.d_background + threadIdx.x, s);
        else
            add_if(G.d_filter_radius, s);
    }
}

__global__ void __launch_bounds__(256, DVG_MINB_INT) k_interior(DevScene S, SampleParams sp, const float* d_render,
                                                                const float* wsum, GradPtrs G, unsigned* status) {
    interior_body<false>(S, sp, sp.tile_base + blockIdx.x, blockIdx.y, d_render, wsum, G, status);
}
__global__ void __launch_bounds__(256, DVG_MINB_LEAN) k_interior_cached(DevScene S, SampleParams sp,
                                                                        const float* d_render, const float* wsum,
                                                                        GradPtrs G, unsigned* status) {
    interior_body<true>(S, sp, sp.tile_base + blockIdx.x, blockIdx.y, d_render, wsum, G, status);
}
__global__ void __launch_bounds__(256, DVG_MINB_INT) k_interior_batch(const BatchEntry* __restrict__ B,
                                                                      const int2* __restrict__ work, int items,
                                                                      int* counter, unsigned* status) {
    for_each_item(items, counter, [&](int i) {
        const int2 wk = work[i];  // (scene, tile + tiles * sub-sample round)
        const BatchEntry& E = B[wk.x];
        const int tiles = E.S.tiles_x * E.S.tiles_y;
        interior_body<false>(E.S, E.sp, wk.y % tiles, wk.y / tiles, E.d_render, E.wsum, E.G, status);
    });
}
__global__ void __launch_bounds__(256, DVG_MINB_LEAN) k_interior_cached_batch(const BatchEntry* __restrict__ B,
                                                                              const int2* __restrict__ work, int items,
                                                                              int* counter, unsigned* status) {
    for_each_item(items, counter, [&](int i) {
        const int2 wk = work[i];  // (scene, tile + tiles * sub-sample round)
        const BatchEntry& E = B[wk.x];
        if (!E.sp.frag) return;  // uniform per item
        const int tiles = E.S.tiles_x * E.S.tiles_y;
        interior_body<true>(E.S, E.sp, wk.y % tiles, wk.y / tiles, E.d_render, E.wsum, E.G, status);
    });
}

// ------------------------------------------------------------------ boundary sampling
// sample_color with an EdgeQuery (sampling.rs:76-224, 485-552) at canvas point pt.
// Returns the un-premultiplied colour (or the premultiplied background when no
// fragment covers pt) and whether the queried shape is the visible boundary.
__device__ float4 edge_color(const DevScene& S, int tile, float2 pt, float4 bg, int eq_group, int eq_shape,
                             bool* hit_out) {
    const int off = S.tile_offsets[tile];
    const int n = S.tile_offsets[tile + 1] - off;
    const int* list = S.tile_entries + off;
    float4 acc = bg;
    int nfrag = 0, ev = 0;  // ev: 0 none, 1 last event sets the hit, 2 last event clears it
    for (int e = 0; e < n; ++e) {
        const int g = __ldg(&list[e]);
        // stroke first, then fill; one paint call site for both
        const int4 gi = __ldg(&S.g_info[g]);
        const float2 lp = xf9(S.g_c2s + 9 * g, pt);
        int hitp[2];
        hitp[0] = gi.y >= 0 && group_within(S, g, lp) ? gi.y : -1;
        hitp[1] = gi.x >= 0 && group_inside(S, g, lp, gi.z) ? gi.x : -1;
#pragma unroll 1
        for (int which = 0; which < 2; ++which) {
            if (hitp[which] < 0) continue;
            const float4 c = paint_color(S, hitp[which], pt);
            over(acc, c);
            ++nfrag;
            if (c.w >= 1.0f) ev = 2;
            if (g == eq_group) ev = 1;
        }
    }
    if (ev != 0) {
        *hit_out = ev == 1;
    } else {  // no deciding fragment: the edge tests on the queried shape alone
              // (within_distance_edge / is_inside_edge)
        bool hit0 = false;
        const int4 gi = __ldg(&S.g_info[eq_group]);
        const float2 lp = xf9(S.g_c2s + 9 * eq_group, pt);
        if (gi.y >= 0) {
            float sw = __ldg(&S.s_stroke[eq_shape]);
            if (sw > 0.0f && within_shape(S, eq_shape, lp, sw)) hit0 = true;
        }
        if (gi.x >= 0) {
            float2 sp = shape_local_bwd(S, eq_shape, lp);
            if (fill_hit(gi.z, winding_shape(S, eq_shape, sp, true))) hit0 = true;
        }
        *hit_out = hit0;
    }
    if (nfrag == 0) return bg;
    float fa = acc.w, fr = acc.x, fg = acc.y, fb = acc.z;
    if (fa > 1.0e-6f) {
        float s = 1.0f / fa;
        fr = fr * s;
        fg = fg * s;
        fb = fb * s;
    }
    return make_float4(fr, fg, fb, fa);
}

__device__ __forceinline__ int lower_bound_cdf(const float* cdf, int n, float u) {
    // first idx with !(u > cdf[idx]) — the crate's linear scan (boundary.rs:454-469)
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (u > __ldg(&cdf[mid]))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
__device__ __forceinline__ float cdf_local_t(const float* cdf, int n, int idx, float u) {
    float prev = idx == 0 ? 0.0f : __ldg(&cdf[idx - 1]);
    float denom = fmaxf(__ldg(&cdf[idx]) - prev, 1.0e-6f);
    return clampf((u - prev) / denom, 0.0f, 1.0f);
}
__device__ __forceinline__ bool path_pt(const DevScene& S, int po, int pc, bool closed, long idx, float2* p) {
    if (pc == 0) return false;
    long i;
    if (closed)
        i = idx % pc;
    else if (idx >= pc)
        return false;
    else
        i = idx;
    *p = S.points[po + i];
    return true;
}
__device__ __forceinline__ bool path_pt_r(const DevScene& S, int po, int pc, bool closed, bool thick, long idx,
                                          float def_r, float2* p, float* r) {
    if (!path_pt(S, po, pc, closed, idx, p)) return false;
    long i = closed ? idx % pc : idx;
    *r = (thick && i < pc) ? S.thickness[po + i] * 1.0f : def_r;
    return true;
}
struct BData {
    int base_point_id, point_id;
    float t;
    bool is_stroke;
};
__device__ __forceinline__ float2 nrm2(float2 v) {
    float l = len2(v.x, v.y);
    return l == 0.0f ? make_float2(0.0f, 0.0f) : make_float2(v.x / l, v.y / l);
}
// Join and cap edges of a stroke with non-round joins or caps (the polygons
// join_cap_hit tests), sampled as part of its boundary: uniform over the sites (the
// non-round joins, and for open paths with non-round caps the two ends), then by
// length along the site's edges.  Like the crate's offset-curve samples, a point
// moves with its centreline point (the vertex): data->point_id is the vertex's path
// point, data->t the radius derivative (p - v) . n / r (every site polygon scales
// about v with the radius), and base_point_id = -1 marks the sample.
__device__ float2 sample_join_cap(const DevScene& S, int path, float t, float2* normal, float* pdf, BData* data) {
    const int4 pi = __ldg(&S.p_info[2 * path]);
    const int4 pi2 = __ldg(&S.p_info[2 * path + 1]);
    const bool closed = pi2.w & PF_CLOSED;
    const int join = (pi2.w >> PF_JOIN_SHIFT) & 3, cap = (pi2.w >> PF_CAP_SHIFT) & 3;
    const int off = pi.x, n = pi.y;
    const int nj = join != JOIN_ROUND ? (closed ? n : n - 1) : 0;
    const int ncap = !closed && cap != CAP_ROUND ? 2 : 0;
    const int sites = nj + ncap;
    if (n <= 0 || sites <= 0) {
        *pdf = 0.0f;
        return make_float2(0, 0);
    }
    int k = (int)(t * (float)sites);
    if (k > sites - 1) k = sites - 1;
    const float u = t * (float)sites - (float)k;
    *pdf /= (float)sites;
    float2 e[4], v;
    int ne = 0, pid = 0;
    float r = 0.0f;
    float2 capdir = make_float2(0, 0);
    if (k < nj) {
        const int vb = closed ? k : k + 1, va = vb > 0 ? vb - 1 : n - 1;
        const float4 a0 = __ldg(&S.seg_p[2 * (off + va)]), a1 = __ldg(&S.seg_p[2 * (off + va) + 1]);
        const float4 b0 = __ldg(&S.seg_p[2 * (off + vb)]), b1 = __ldg(&S.seg_p[2 * (off + vb) + 1]);
        v = make_float2(b0.x, b0.y);
        r = __ldg(&S.seg_r[off + vb]).x;
        pid = __ldg(&S.seg_meta[off + vb]).z;
        float2 din = seg_dir1(a0, a1), dout = seg_dir0(b0, b1);
        const float li = sqrtf(din.x * din.x + din.y * din.y), lo = sqrtf(dout.x * dout.x + dout.y * dout.y);
        if (!(li > 0.0f) || !(lo > 0.0f) || !(r > 0.0f)) {
            *pdf = 0.0f;
            return make_float2(0, 0);
        }
        din = make_float2(din.x / li, din.y / li);
        dout = make_float2(dout.x / lo, dout.y / lo);
        const float cr = cross2f(din.x, din.y, dout.x, dout.y);
        if (fabsf(cr) < 1.0e-6f) {  // no outer corner: no edge here
            *pdf = 0.0f;
            return make_float2(0, 0);
        }
        const float sg = cr > 0.0f ? 1.0f : -1.0f;
        e[0] = make_float2(v.x + r * sg * din.y, v.y - r * sg * din.x);
        const float2 b = make_float2(v.x + r * sg * dout.y, v.y - r * sg * dout.x);
        ne = 1;
        if (join == JOIN_MITER) {
            const float sm = cross2f(b.x - e[0].x, b.y - e[0].y, dout.x, dout.y) / cr;
            const float2 m = make_float2(e[0].x + sm * din.x, e[0].y + sm * din.y);
            const float ml = sqrtf((m.x - v.x) * (m.x - v.x) + (m.y - v.y) * (m.y - v.y));
            if (ml <= __ldg(&S.p_miter[path]) * r) e[ne++] = m;
        }
        e[ne] = b;
    } else {
        const bool start = k == nj;
        const int sidx = start ? 0 : n - 1;
        const float4 q0 = __ldg(&S.seg_p[2 * (off + sidx)]), q1 = __ldg(&S.seg_p[2 * (off + sidx) + 1]);
        float2 d;
        if (start) {
            const float2 d0 = seg_dir0(q0, q1);
            d = make_float2(-d0.x, -d0.y);
            v = make_float2(q0.x, q0.y);
            r = __ldg(&S.seg_r[off]).x;
            pid = __ldg(&S.seg_meta[off]).z;
        } else {
            d = seg_dir1(q0, q1);
            v = make_float2(q1.z, q1.w);
            r = __ldg(&S.seg_r[off + n - 1]).w;
            pid = pi2.y - 1;
        }
        const float l = sqrtf(d.x * d.x + d.y * d.y);
        if (!(l > 0.0f) || !(r > 0.0f)) {
            *pdf = 0.0f;
            return make_float2(0, 0);
        }
        d = make_float2(d.x / l, d.y / l);
        capdir = d;
        const float2 np = make_float2(-d.y, d.x);
        e[0] = make_float2(v.x - r * np.x, v.y - r * np.y);
        if (cap == CAP_SQUARE) {
            e[1] = make_float2(e[0].x + r * d.x, e[0].y + r * d.y);
            e[2] = make_float2(v.x + r * np.x + r * d.x, v.y + r * np.y + r * d.y);
            e[3] = make_float2(v.x + r * np.x, v.y + r * np.y);
            ne = 3;
        } else {
            e[1] = make_float2(v.x + r * np.x, v.y + r * np.y);
            ne = 1;
        }
    }
    float len[3], total = 0.0f;
    for (int i = 0; i < ne; ++i) {
        len[i] = len2(e[i + 1].x - e[i].x, e[i + 1].y - e[i].y);
        total += len[i];
    }
    if (!(total > 0.0f)) {
        *pdf = 0.0f;
        return make_float2(0, 0);
    }
    float sl = u * total;
    int i = 0;
    while (i < ne - 1 && sl > len[i]) sl -= len[i++];
    const float f = len[i] > 0.0f ? fminf(sl / len[i], 1.0f) : 0.0f;
    const float2 p = make_float2(e[i].x + f * (e[i + 1].x - e[i].x), e[i].y + f * (e[i + 1].y - e[i].y));
    float2 nn = nrm2(make_float2(-(e[i + 1].y - e[i].y), e[i + 1].x - e[i].x));
    const float mx = 0.5f * (e[i].x + e[i + 1].x) - v.x, my = 0.5f * (e[i].y + e[i + 1].y) - v.y;
    const float side = (mx == 0.0f && my == 0.0f) ? nn.x * capdir.x + nn.y * capdir.y : nn.x * mx + nn.y * my;
    if (side < 0.0f) nn = make_float2(-nn.x, -nn.y);
    *pdf /= total;
    *normal = nn;
    (void)pid;
    data->base_point_id = -1 - k;  // the site
    data->point_id = i;            // the edge of the site's polygon
    data->t = f;                   // the position along that edge
    return p;
}

// Normal velocity of the join / cap edge point sampled at (site, edge, f):
// w[k] = dp/dtheta_k . n for theta = (v, qa, qb, r); ids = path points of v, qa, qb
// (-1: not used).  Out of line: it runs only for those samples.
static __device__ __noinline__ bool join_cap_velocity(const int4* p_info, const float* p_miter, const float4* seg_p,
                                                     const float4* seg_r, const int4* seg_meta, int path, int site,
                                                     int edge, float f, float nx, float ny, float* w, int* ids) {
    const int4 pi = __ldg(&p_info[2 * path]);
    const int4 pi2 = __ldg(&p_info[2 * path + 1]);
    const bool closed = pi2.w & PF_CLOSED;
    const int join = (pi2.w >> PF_JOIN_SHIFT) & 3, cap = (pi2.w >> PF_CAP_SHIFT) & 3;
    const int off = pi.x, nseg = pi.y, pc = pi2.y;
    const int nj = join != JOIN_ROUND ? (closed ? nseg : nseg - 1) : 0;
    ids[0] = ids[1] = ids[2] = -1;
    DV e[4];
    int ne = 0;
    if (site < nj) {
        const int vb = closed ? site : site + 1, va = vb > 0 ? vb - 1 : nseg - 1;
        const float4 a0 = __ldg(&seg_p[2 * (off + va)]), a1 = __ldg(&seg_p[2 * (off + va) + 1]);
        const float4 b0 = __ldg(&seg_p[2 * (off + vb)]), b1 = __ldg(&seg_p[2 * (off + vb) + 1]);
        const int sa = seg_dir1_slot(a0, a1), sb = seg_dir0_slot(b0, b1);
        const float2 v = make_float2(b0.x, b0.y), qa = seg_slot(a0, a1, sa), qb = seg_slot(b0, b1, sb);
        const int4 ma = __ldg(&seg_meta[off + va]), mb = __ldg(&seg_meta[off + vb]);
        ids[0] = mb.z;
        ids[1] = seg_slot_point(ma, sa, closed, pc);
        ids[2] = seg_slot_point(mb, sb, closed, pc);
        const DV V{dl_var(v.x, 0), dl_var(v.y, 1)}, QA{dl_var(qa.x, 2), dl_var(qa.y, 3)},
            QB{dl_var(qb.x, 4), dl_var(qb.y, 5)};
        const Dl R = dl_var(__ldg(&seg_r[off + vb]).x, 6);
        const DV din = dv_unit(dv_sub(V, QA)), dout = dv_unit(dv_sub(QB, V));
        const Dl cr = din.x * dout.y - din.y * dout.x;
        if (fabsf(cr.v) < 1.0e-6f) return false;
        const Dl sg = dl_const(cr.v > 0.0f ? 1.0f : -1.0f);
        e[0] = DV{V.x + R * sg * din.y, V.y - R * sg * din.x};
        const DV b{V.x + R * sg * dout.y, V.y - R * sg * dout.x};
        ne = 1;
        if (join == JOIN_MITER) {
            const Dl sm = ((b.x - e[0].x) * dout.y - (b.y - e[0].y) * dout.x) / cr;
            const DV m = dv_add(e[0], dv_scale(din, sm));
            const float ml = sqrtf((m.x.v - v.x) * (m.x.v - v.x) + (m.y.v - v.y) * (m.y.v - v.y));
            if (ml <= __ldg(&p_miter[path]) * R.v) e[ne++] = m;
        }
        e[ne] = b;
    } else {
        const bool start = site == nj;
        const int si = start ? 0 : nseg - 1;
        const float4 q0 = __ldg(&seg_p[2 * (off + si)]), q1 = __ldg(&seg_p[2 * (off + si) + 1]);
        const int sq = start ? seg_dir0_slot(q0, q1) : seg_dir1_slot(q0, q1);
        const float2 v = start ? make_float2(q0.x, q0.y) : make_float2(q1.z, q1.w), q = seg_slot(q0, q1, sq);
        const int4 m = __ldg(&seg_meta[off + si]);
        ids[0] = start ? m.z : pc - 1;
        ids[start ? 2 : 1] = seg_slot_point(m, sq, closed, pc);
        const DV V{dl_var(v.x, 0), dl_var(v.y, 1)};
        const DV Q = start ? DV{dl_var(q.x, 4), dl_var(q.y, 5)} : DV{dl_var(q.x, 2), dl_var(q.y, 3)};
        const float4 rr = __ldg(&seg_r[off + si]);
        const Dl R = dl_var(start ? rr.x : rr.w, 6);
        const DV d = dv_unit(dv_sub(V, Q));  // outward along the end
        const DV np{dl_const(0.0f) - d.y, d.x};
        e[0] = dv_sub(V, dv_scale(np, R));
        if (cap == CAP_SQUARE) {
            e[1] = dv_add(e[0], dv_scale(d, R));
            e[2] = dv_add(dv_add(V, dv_scale(np, R)), dv_scale(d, R));
            e[3] = dv_add(V, dv_scale(np, R));
            ne = 3;
        } else {
            e[1] = dv_add(V, dv_scale(np, R));
            ne = 1;
        }
    }
    if (edge >= ne) return false;
    const DV p = dv_add(e[edge], dv_scale(dv_sub(e[edge + 1], e[edge]), dl_const(f)));
#pragma unroll
    for (int k = 0; k < 7; ++k) w[k] = p.x.d[k] * nx + p.y.d[k] * ny;
    return true;
}

// sample_boundary_path (boundary.rs:630-842)
__device__ float2 sample_boundary_path(const DevScene& S, int shape, float path_len, float t, float2* normal,
                                       float* pdf, BData* data, float dir, float srad) {
    const int path = __ldg(&S.s_info[shape].z);
    const int4 pi2 = __ldg(&S.p_info[2 * path + 1]);
    const int po = pi2.x, pc = pi2.y, co = pi2.z;
    const bool closed = pi2.w & PF_CLOSED;
    const bool thick = pi2.w & PF_THICK;
    const int4 cinfo = __ldg(&S.path_cdf_info[shape]);
    const int nb = cinfo.y;
    if (pc == 0 || nb == 0) {
        *pdf = 0.0f;
        return make_float2(0, 0);
    }
    const bool styled = dir != 0.0f && (pi2.w & PF_STYLED);
    if (styled) {  // a share of the samples on the join / cap edges (both sides draw them)
        const float q = JOIN_CAP_SHARE;
        if (t < q) {
            *pdf *= 2.0f * q;
            return sample_join_cap(S, path, t / q, normal, pdf, data);
        }
        t = (t - q) / (1.0f - q);
        *pdf *= 1.0f - q;
    }
    if (dir != 0.0f && !closed && (!styled || ((pi2.w >> PF_CAP_SHIFT) & 3) == CAP_ROUND)) {
        float cap = 0.0f;
        if (thick)
            cap = PI_F * (S.thickness[po] + S.thickness[po + pc - 1]);
        else
            cap = 2.0f * PI_F * srad;
        float denom = cap + path_len;
        if (denom > 0.0f) {
            float cp = cap / denom;
            if (t < cp) {
                t /= cp;
                *pdf *= cp;
                float r0 = srad, r1 = srad;
                if (thick) {
                    r0 = S.thickness[po];
                    r1 = S.thickness[po + pc - 1];
                }
                float ang = 2.0f * PI_F * t;
                if (dir < 0.0f) {
                    float2 o = make_float2(r0 * dvg_cosf(ang), r0 * dvg_sinf(ang));
                    *normal = nrm2(o);
                    *pdf /= 2.0f * PI_F * r0;
                    data->base_point_id = 0;
                    data->point_id = 0;
                    data->t = 0.0f;
                    float2 p0 = S.points[po];
                    return make_float2(p0.x + o.x, p0.y + o.y);
                }
                float2 o = make_float2(r1 * dvg_cosf(ang), r1 * dvg_sinf(ang));
                *normal = nrm2(o);
                *pdf /= 2.0f * PI_F * r1;
                data->base_point_id = nb - 1;
                int controls = S.ncp[co + nb - 1];
                data->point_id = pc >= 2 + controls ? pc - (2 + controls) : 0;
                data->t = 1.0f;
                float2 pl = S.points[po + pc - 1];
                return make_float2(pl.x + o.x, pl.y + o.y);
            }
            t = (t - cp) / (1.0f - cp);
            *pdf *= 1.0f - cp;
        }
    }
    const float* cdf = S.path_cdf + cinfo.x;
    int sid = lower_bound_cdf(cdf, nb, t);
    if (sid >= nb) sid = nb - 1;
    float lt = cdf_local_t(cdf, nb, sid, t);
    int pid = S.path_pid[cinfo.x + sid];
    data->base_point_id = sid;
    data->point_id = pid;
    data->t = lt;
    if (lt < -1.0e-3f || lt > 1.0f + 1.0e-3f) {
        *pdf = 0.0f;
        return make_float2(0, 0);
    }
    int nc = S.ncp[co + sid];
    float pmf = S.path_pmf[cinfo.x + sid];
    auto nxt = [&](long i) -> long { return closed ? i % pc : (i < pc - 1 ? i : pc - 1); };
    float2 q[4];
    float r[4];
    int np = nc + 2;
    if (nc > 2) {
        *pdf = 0.0f;
        return make_float2(0, 0);
    }
    for (int k = 0; k < np; ++k) {
        long idx = (k == np - 1) ? nxt(pid + k) : (long)(pid + k);
        if (!path_pt_r(S, po, pc, closed, thick, idx, srad, &q[k], &r[k])) {
            *pdf = 0.0f;
            return make_float2(0, 0);
        }
    }
    float tt = 1.0f - lt;
    float2 ev, tg;
    float rr;
    if (nc == 0) {
        tg = make_float2(q[1].x - q[0].x, q[1].y - q[0].y);
        ev = make_float2(q[0].x + tg.x * lt, q[0].y + tg.y * lt);
        rr = r[0] + lt * (r[1] - r[0]);
    } else if (nc == 1) {
        float w0 = tt * tt, w1 = 2.0f * tt * lt, w2 = lt * lt;
        ev = make_float2(q[0].x * w0 + q[1].x * w1 + q[2].x * w2, q[0].y * w0 + q[1].y * w1 + q[2].y * w2);
        float a = 2.0f * tt, b = 2.0f * lt;
        tg = make_float2((q[1].x - q[0].x) * a + (q[2].x - q[1].x) * b, (q[1].y - q[0].y) * a + (q[2].y - q[1].y) * b);
        rr = r[0] * w0 + r[1] * w1 + r[2] * w2;
    } else {
        float w0 = tt * tt * tt, w1 = 3.0f * tt * tt * lt, w2 = 3.0f * tt * lt * lt, w3 = lt * lt * lt;
        ev = make_float2(q[0].x * w0 + q[1].x * w1 + q[2].x * w2 + q[3].x * w3,
                         q[0].y * w0 + q[1].y * w1 + q[2].y * w2 + q[3].y * w3);
        float a = 3.0f * tt * tt, b = 6.0f * tt * lt, c = 3.0f * lt * lt;
        tg = make_float2((q[1].x - q[0].x) * a + (q[2].x - q[1].x) * b + (q[3].x - q[2].x) * c,
                         (q[1].y - q[0].y) * a + (q[2].y - q[1].y) * b + (q[3].y - q[2].y) * c);
        rr = r[0] * w0 + r[1] * w1 + r[2] * w2 + r[3] * w3;
    }
    float tl = len2(tg.x, tg.y);
    if (tl == 0.0f) {
        *pdf = 0.0f;
        return make_float2(0, 0);
    }
    *normal = make_float2(-tg.y / tl, tg.x / tl);
    *pdf *= pmf / tl;
    if (dir != 0.0f) {
        ev.x += normal->x * (dir * rr);
        ev.y += normal->y * (dir * rr);
        if (dir < 0.0f) *normal = make_float2(normal->x * -1.0f, normal->y * -1.0f);
    }
    return ev;
}
// sample_boundary_point (boundary.rs:472-627)
__device__ bool sample_boundary_point(const DevScene& S, int shape, int group, float t, float shape_len,
                                      float2* pt_out, float2* normal_out, float* pdf_out, BData* data) {
    const int4 gi = __ldg(&S.g_info[group]);
    const bool has_fill = gi.x >= 0, has_stroke = gi.y >= 0;
    if (!has_fill && !has_stroke) return false;
    float pdf = 1.0f, lt = t;
    bool stroke = false;
    if (has_fill && has_stroke) {
        if (lt < 0.5f) {
            lt *= 2.0f;
        } else {
            stroke = true;
            lt = 2.0f * (lt - 0.5f);
        }
        pdf = 0.5f;
    } else if (has_stroke) {
        stroke = true;
    }
    float dir = 0.0f;
    if (stroke) {
        if (lt < 0.5f) {
            dir = -1.0f;
            lt *= 2.0f;
        } else {
            dir = 1.0f;
            lt = 2.0f * (lt - 0.5f);
        }
        pdf *= 0.5f;
    }
    data->base_point_id = 0;
    data->point_id = 0;
    data->t = 0.0f;
    data->is_stroke = stroke;
    const int4 si = __ldg(&S.s_info[shape]);
    const float4 prm = __ldg(&S.s_params[shape]);
    const float sw = __ldg(&S.s_stroke[shape]);
    float2 normal = make_float2(0, 0), out;
    if (si.x == K_CIRCLE) {
        float r = fabsf(prm.z);
        if (r <= 0.0f) return false;
        float ang = 2.0f * PI_F * lt;
        float2 o = make_float2(r * dvg_cosf(ang), r * dvg_sinf(ang));
        normal = nrm2(o);
        pdf /= 2.0f * PI_F * r;
        out = make_float2(prm.x + o.x, prm.y + o.y);
    } else if (si.x == K_ELLIPSE) {
        float rx = fabsf(prm.z), ry = fabsf(prm.w);
        if (rx <= 0.0f || ry <= 0.0f) return false;
        float ang = 2.0f * PI_F * lt;
        float s = dvg_sinf(ang), c = dvg_cosf(ang);
        float dxdt = -rx * s * 2.0f * PI_F, dydt = ry * c * 2.0f * PI_F;
        normal = nrm2(make_float2(dydt, -dxdt));
        pdf /= sqrtf(dxdt * dxdt + dydt * dydt);
        out = make_float2(prm.x + rx * c, prm.y + ry * s);
    } else if (si.x == K_RECT) {
        float w = prm.z - prm.x, h = prm.w - prm.y;
        if (w == 0.0f && h == 0.0f) return false;
        pdf /= 2.0f * (w + h);
        if (lt <= w / (w + h)) {
            lt *= (w + h) / w;
            if (lt < 0.5f) {
                normal = make_float2(0.0f, -1.0f);
                out = make_float2(prm.x + 2.0f * lt * (prm.z - prm.x), prm.y + 0.0f);
            } else {
                normal = make_float2(0.0f, 1.0f);
                out = make_float2(prm.x + 2.0f * (lt - 0.5f) * (prm.z - prm.x), prm.w + 0.0f);
            }
        } else {
            lt = (lt - w / (w + h)) * (w + h) / h;
            if (lt < 0.5f) {
                normal = make_float2(-1.0f, 0.0f);
                out = make_float2(prm.x + 0.0f, prm.y + 2.0f * lt * (prm.w - prm.y));
            } else {
                normal = make_float2(1.0f, 0.0f);
                out = make_float2(prm.z + 0.0f, prm.y + 2.0f * (lt - 0.5f) * (prm.w - prm.y));
            }
        }
    } else {
        if (si.z < 0) return false;
        const int4 ci = __ldg(&S.path_cdf_info[shape]);
        if (!ci.z) return false;
        if (S.path_len[shape] <= 0.0f) return false;
        out = sample_boundary_path(S, shape, shape_len, lt, &normal, &pdf, data, dir, sw);
        dir = 0.0f;  // the path sampler applies the stroke offset itself
    }
    if (dir != 0.0f) {
        out.x += normal.x * (dir * sw);
        out.y += normal.y * (dir * sw);
        if (dir < 0.0f) normal = make_float2(normal.x * -1.0f, normal.y * -1.0f);
    }
    if (!isfinite(pdf) || pdf <= 0.0f) return false;
    *pt_out = out;
    *normal_out = normal;
    *pdf_out = pdf;
    return true;
}
// The gradient of one join / cap edge sample (out of line with scalar arguments: the
// boundary kernel is instruction-fetch bound and these samples are few).
static __device__ __noinline__ void accumulate_join_cap(const int4* p_info, const float* p_miter,
                                                       const float4* seg_p, const float4* seg_r,
                                                       const int4* seg_meta, float* d_points, float* d_thickness,
                                                       float* d_stroke_width, int path, int po, int site, int edge,
                                                       float f, float nx, float ny, float contrib) {
    float w[7];
    int ids[3];
    if (!join_cap_velocity(p_info, p_miter, seg_p, seg_r, seg_meta, path, site, edge, f, nx, ny, w, ids)) return;
    for (int j = 0; j < 3; ++j)
        if (ids[j] >= 0) {
            add_if(d_points + 2 * (po + ids[j]), w[2 * j] * contrib);
            add_if(d_points + 2 * (po + ids[j]) + 1, w[2 * j + 1] * contrib);
        }
    if (d_thickness)
        add_if(d_thickness + po + ids[0], w[6] * contrib);
    else
        add_if(d_stroke_width, w[6] * contrib);
}
__device__ __forceinline__ void mul33(const float* a, const float* b, float* o) {  // Mat3::mul
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) o[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
}
// accumulate_boundary_gradient (boundary.rs:970-1148)
// STYLED: the scene has strokes with non-round joins or caps (join / cap edge samples,
// base_point_id < 0); the kernels of other scenes carry none of that code.
template <bool STYLED>
__device__ void accumulate_boundary(const DevScene& S, const GradPtrs& G, int shape, int group, float contrib,
                                    float t, float2 n, const BData& bd, float2 local_pt) {
    const int4 si = __ldg(&S.s_info[shape]);
    int po = 0, pc = 0, co = 0, pflags = 0;
    if (si.x == K_PATH && si.z >= 0) {
        int4 pi2 = __ldg(&S.p_info[2 * si.z + 1]);
        po = pi2.x;
        pc = pi2.y;
        co = pi2.z;
        pflags = pi2.w;
    }
    const bool closed = pflags & PF_CLOSED;
    int nc = 0;  // num_control_points.get(base_point_id).unwrap_or(0)
    if (si.x == K_PATH && (!STYLED || bd.base_point_id >= 0)) {
        int ctrl_count = __ldg(&S.path_cdf_info[shape].y);
        nc = bd.base_point_id < ctrl_count ? S.ncp[co + bd.base_point_id] : 0;
    }
    if (STYLED && bd.base_point_id < 0) {  // a join / cap edge sample: the exact normal velocity
        accumulate_join_cap(S.p_info, S.p_miter, S.seg_p, S.seg_r, S.seg_meta, G.d_points,
                            (pflags & PF_THICK) ? G.d_thickness : nullptr, G.d_shape_stroke_width + shape, si.z, po,
                            -1 - bd.base_point_id, bd.point_id, bd.t, n.x, n.y, contrib);
    } else if (bd.is_stroke) {
        if (si.x == K_PATH && (pflags & PF_THICK)) {
            float t2 = bd.t, tt = 1.0f - t2;
            int pid = bd.point_id;
            auto addt = [&](long i, float v) {
                if (i < pc) add_if(G.d_thickness + po + i, v);
            };
            if (nc == 0) {
                addt(pid, (1.0f - t2) * contrib);
                addt(closed ? (pid + 1) % pc : pid + 1, t2 * contrib);
            } else if (nc == 1) {
                addt(pid, tt * tt * contrib);
                addt(pid + 1, 2.0f * tt * t2 * contrib);
                addt(closed ? (pid + 2) % pc : pid + 2, t2 * t2 * contrib);
            } else if (nc == 2) {
                addt(pid, tt * tt * tt * contrib);
                addt(pid + 1, 3.0f * tt * tt * t2 * contrib);
                addt(pid + 2, 3.0f * tt * t2 * t2 * contrib);
                addt(closed ? (pid + 3) % pc : pid + 3, t2 * t2 * t2 * contrib);
            }
        } else {
            add_if(G.d_shape_stroke_width + shape, contrib);
        }
    }
    float* dp = G.d_shape_params + 4 * shape;
    if (si.x == K_CIRCLE) {
        add_if(dp + 0, n.x * contrib);
        add_if(dp + 1, n.y * contrib);
        add_if(dp + 2, contrib);
    } else if (si.x == K_ELLIPSE) {
        add_if(dp + 0, n.x * contrib);
        add_if(dp + 1, n.y * contrib);
        float ang = 2.0f * PI_F * t;
        add_if(dp + 2, dvg_cosf(ang) * n.x * contrib);
        add_if(dp + 3, dvg_sinf(ang) * n.y * contrib);
    } else if (si.x == K_PATH && (!STYLED || bd.base_point_id >= 0)) {
        float t2 = bd.t, tt = 1.0f - t2;
        int pid = bd.point_id;
        auto addp = [&](long idx, float w) {
            long i = closed ? idx % pc : idx;
            if (i < pc) {
                add_if(G.d_points + 2 * (po + i), n.x * (w * contrib));
                add_if(G.d_points + 2 * (po + i) + 1, n.y * (w * contrib));
            }
        };
        if (nc == 0) {
            addp(pid, 1.0f - t2);
            addp(pid + 1, t2);
        } else if (nc == 1) {
            addp(pid, tt * tt);
            addp(pid + 1, 2.0f * tt * t2);
            addp(pid + 2, t2 * t2);
        } else if (nc == 2) {
            addp(pid, tt * tt * tt);
            addp(pid + 1, 3.0f * tt * tt * t2);
            addp(pid + 2, 3.0f * tt * t2 * t2);
            addp(pid + 3, t2 * t2 * t2);
        }
    } else if (si.x == K_RECT) {
        if (n.x == -1.0f && n.y == 0.0f)
            add_if(dp + 0, -contrib);
        else if (n.x == 1.0f && n.y == 0.0f)
            add_if(dp + 2, contrib);
        else if (n.x == 0.0f && n.y == -1.0f)
            add_if(dp + 1, -contrib);
        else if (n.x == 0.0f && n.y == 1.0f)
            add_if(dp + 3, contrib);
    }
    // transforms (boundary.rs:1132-1147) with d_xform_pt (backward/math.rs:109-128)
    const float* gs = S.g_s2c + 9 * group;
    const float* sx = S.s_xform + 9 * shape;
    float m[9];
    mul33(gs, sx, m);
    const float2 dout = make_float2(n.x * contrib, n.y * contrib);
    const float2 p = local_pt;
    float t0 = m[0] * p.x + m[1] * p.y + m[2];
    float t1 = m[3] * p.x + m[4] * p.y + m[5];
    float t2 = m[6] * p.x + m[7] * p.y + m[8];
    float ox = t0 / t2, oy = t1 / t2;
    float d0 = dout.x / t2, d1 = dout.y / t2, d2 = -(dout.x * ox + dout.y * oy) / t2;
    float dm[9] = {d0 * p.x, d0 * p.y, d0, d1 * p.x, d1 * p.y, d1, d2 * p.x, d2 * p.y, d2};
    // d_group = dm * shape_xform^T ; d_shape = group_s2c^T * dm
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float dg = dm[3 * r] * sx[3 * c] + dm[3 * r + 1] * sx[3 * c + 1] + dm[3 * r + 2] * sx[3 * c + 2];
            float ds = gs[r] * dm[c] + gs[3 + r] * dm[3 + c] + gs[6 + r] * dm[6 + c];
            add_if(G.d_group_transform + 9 * group + 3 * r + c, dg);
            add_if(G.d_shape_transform + 9 * shape + 3 * r + c, ds);
        }
}

// Boundary pass, stage 1: draw every edge sample (boundary.rs:141-175), keep
// the valid ones with the tile of their boundary pixel as sort key.
__device__ __forceinline__ void boundary_gen_one(const DevScene& S, uint64_t idx, uint64_t slot, uint32_t seed,
                                                 int rng_kind, int tile_off, int scene, int cell, float pdf_scale,
                                                 BSample* out, int* key, int* tile_counts) {
    key[slot] = -1;
    float u, t;
    if (rng_kind == 1) {
        uint4 r = philox4x32_10(make_uint4((uint32_t)idx, (uint32_t)(idx >> 32), 0u, 0u), make_uint2(seed, 0u));
        u = unit_from_u32(r.x);
        t = unit_from_u32(r.y);
    } else {
        Pcg32 rng(idx, (uint64_t)seed);
        u = rng.next_f32();
        t = rng.next_f32();
    }
    int sid = lower_bound_cdf(S.bcdf, S.bcdf_n, u);
    if (sid >= S.bcdf_n) sid = S.bcdf_n - 1;
    const int shape = S.b_shape[sid], group = S.b_group[sid];
    const float pmf = S.bpmf[sid];
    if (pmf <= 0.0f) return;
    float2 local_pt, normal;
    float bpdf;
    BData bd;
    if (!sample_boundary_point(S, shape, group, t, S.shape_len[shape], &local_pt, &normal, &bpdf, &bd)) return;
    if (bpdf <= 0.0f) return;
    float s2c[9];
    mul33(S.g_s2c + 9 * group, S.s_xform + 9 * shape, s2c);
    float2 bpt = xf9(s2c, local_pt);
    float sinv[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (__ldg(&S.s_info[shape].y) & SF_INVERTIBLE) {
        const float* iv = S.s_inv + 6 * shape;
        for (int k = 0; k < 6; ++k) sinv[k] = iv[k];
    }
    float cinv[9];
    mul33(sinv, S.g_c2s + 9 * group, cinv);
    float2 nc = nrm2(make_float2(cinv[0] * normal.x + cinv[3] * normal.y, cinv[1] * normal.x + cinv[4] * normal.y));
    const float W = (float)S.width, H = (float)S.height;
    bpt.x /= W;
    bpt.y /= H;
    const float pdf = pmf * bpdf * pdf_scale;
    if (pdf <= 0.0f) return;
    const int bx = f2i(bpt.x * W), by = f2i(bpt.y * H);
    if (bx < 0 || bx >= S.width || by < 0 || by >= S.height) return;
    BSample r;
    r.bx = bpt.x;
    r.by = bpt.y;
    r.nx = nc.x;
    r.ny = nc.y;
    r.lx = local_pt.x;
    r.ly = local_pt.y;
    r.pdf = pdf;
    r.t = t;
    r.shape = shape;
    r.group = group;
    r.pixel = by * S.width + bx;
    r.base_point_id = bd.base_point_id;
    r.point_id = bd.point_id;
    r.bt = bd.t;
    r.is_stroke = bd.is_stroke ? 1 : 0;
    r.scene = scene;
    out[slot] = r;
    // sort bucket: the cell of the boundary pixel inside its tile, so that a warp
    // evaluates edge points that lie close together (coherent group walks), then the
    // sample's class, so that it mostly runs one sampling / gradient code path
    const int tile = tile_off + (by / TILE) * S.tiles_x + (bx / TILE);
    const int per_row = TILE / cell;
    const int cls = (bd.is_stroke ? 2 : 0) + (__ldg(&S.s_info[shape]).x == K_PATH ? 1 : 0);
    const int bucket =
        (tile * (per_row * per_row) + ((by % TILE) / cell) * per_row + (bx % TILE) / cell) * BND_CLASSES + cls;
    key[slot] = bucket;
    atomicAdd(tile_counts + bucket, 1);
}
__global__ void __launch_bounds__(256) k_boundary_gen(DevScene S, BoundaryParams bp, BSample* out, int* key,
                                                      int* tile_counts) {
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + bp.sample_base;
    if (idx >= bp.num_samples) return;
    boundary_gen_one(S, idx, idx - bp.slot_base, bp.seed, bp.rng, 0, 0, bp.cell, bp.pdf_scale, out, key,
                     tile_counts);
}
// Batched stage 1: one flat index over all scenes' boundary samples; the scene is
// found by binary search over the per-scene sample offsets.
__global__ void __launch_bounds__(256) k_boundary_gen_batch(const BatchEntry* __restrict__ B, int nscenes,
                                                            uint64_t total, int cell, BSample* out, int* key,
                                                            int* tile_counts) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int lo = 0, hi = nscenes - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (B[mid].b_off <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    const BatchEntry& E = B[lo];
    key[g] = -1;
    if (!E.S.boundary_ok || g - E.b_off >= E.nb) return;
    boundary_gen_one(E.S, g - E.b_off, g, E.bseed, E.rng, E.tile_off, lo, cell, E.bscale, out, key, tile_counts);
}
// Stage 2: counting-sort scatter of sample slots by tile.
__global__ void k_boundary_scatter(const int* key, uint64_t n, int* cursor, int* order) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = key[i];
    if (k < 0) return;
    order[atomicAdd(cursor + k, 1)] = (int)i;
}
// Stage 3: evaluate both sides of every edge sample in tile order, so that the
// lanes of a warp share one group list (render_edge_sample, boundary.rs:845-967).
// Two lanes per sample: the even lane of a pair takes the colour inside, the odd lane
// the colour outside.  The two points are 2e-4 of the canvas apart, so a pair walks
// the same BVH nodes and segment tests in lockstep; the even lane receives the odd
// lane's colour and hit by shuffle and finishes the sample alone.  Every lane of the
// warp reaches the shuffles (`valid` false: a pair past the last sample).
template <bool STYLED>
__device__ __forceinline__ void boundary_eval_pair(const DevScene& S, const BSample& r, bool valid,
                                                   const float* d_render, const float* wsum, const GradPtrs& G) {
    const float W = (float)S.width, H = (float)S.height;
    const int side = threadIdx.x & 1;
    float4 cs = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    bool hs = false;
    float4 bg = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (valid) {
        bg = background_premul(S, r.pixel);
        const int tile = ((r.pixel / S.width) / TILE) * S.tiles_x + ((r.pixel % S.width) / TILE);
        const float o = side == 0 ? -1.0e-4f : 1.0e-4f;
        const float2 q = make_float2(r.bx + r.nx * o, r.by + r.ny * o);
        cs = edge_color(S, tile, make_float2(q.x * W, q.y * H), bg, r.group, r.shape, &hs);
    }
    float4 co;
    co.x = __shfl_xor_sync(0xffffffffu, cs.x, 1);
    co.y = __shfl_xor_sync(0xffffffffu, cs.y, 1);
    co.z = __shfl_xor_sync(0xffffffffu, cs.z, 1);
    co.w = __shfl_xor_sync(0xffffffffu, cs.w, 1);
    const bool ho = __shfl_xor_sync(0xffffffffu, (int)hs, 1) != 0;
    if (!valid || side != 0) return;
    float2 nc = make_float2(r.nx, r.ny);
    float4 ci = cs;
    const bool hi = hs;
    if (!hi && !ho) return;
    if (!hi) {
        nc = make_float2(nc.x * -1.0f, nc.y * -1.0f);
        float4 tmp = ci;
        ci = co;
        co = tmp;
    }
    // gather_d_color at the boundary pixel, divided by W*H (boundary.rs:913-929)
    const float2 sb = make_float2(r.bx * W, r.by * H);
    float4 dc = make_float4(0, 0, 0, 0);
    {
        const int px = f2i(floorf(sb.x)), py = f2i(floorf(sb.y)), ri = S.filter_ri;
        for (int dy = -ri; dy <= ri; ++dy)
            for (int dx = -ri; dx <= ri; ++dx) {
                int xx = px + dx, yy = py + dy;
                if (xx < 0 || yy < 0 || xx >= S.width || yy >= S.height) continue;
                float w = filter_weight(S.filter_type, S.filter_radius, (float)xx + 0.5f - sb.x,
                                        (float)yy + 0.5f - sb.y);
                size_t q = (size_t)yy * S.width + xx;
                float ws = wsum[q];
                if (ws > 0.0f) {
                    float4 d = reinterpret_cast<const float4*>(d_render)[q];
                    float k = w / ws;
                    dc.x += k * d.x;
                    dc.y += k * d.y;
                    dc.z += k * d.z;
                    dc.w += k * d.w;
                }
            }
    }
    const float norm = W * H;
    if (norm > 0.0f) {
        dc.x /= norm;
        dc.y /= norm;
        dc.z /= norm;
        dc.w /= norm;
    }
    const float contrib =
        ((ci.x - co.x) * dc.x + (ci.y - co.y) * dc.y + (ci.z - co.z) * dc.z + (ci.w - co.w) * dc.w) / r.pdf;
    if (!isfinite(contrib)) return;
    BData bd;
    bd.base_point_id = r.base_point_id;
    bd.point_id = r.point_id;
    bd.t = r.bt;
    bd.is_stroke = r.is_stroke != 0;
    accumulate_boundary<STYLED>(S, G, r.shape, r.group, contrib, r.t, nc, bd, make_float2(r.lx, r.ly));
    if (G.d_translation) {
        add_if(G.d_translation + 2 * (size_t)r.pixel, nc.x * contrib);
        add_if(G.d_translation + 2 * (size_t)r.pixel + 1, nc.y * contrib);
    }
}
// Two threads per sample (boundary_eval_pair): launch 2 * samples threads.
template <bool STYLED>
__global__ void __launch_bounds__(128, DVG_MINB_BND) k_boundary_eval(DevScene S, const BSample* samples,
                                                                     const int* order, const int* offsets, int tiles,
                                                                     const float* d_render, const float* wsum,
                                                                     GradPtrs G) {
    const int64_t i = (int64_t)(((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 1);
    const bool valid = i < offsets[tiles];
    BSample r{};
    if (valid) r = samples[order[i]];
    boundary_eval_pair<STYLED>(S, r, valid, d_render, wsum, G);
}
template <bool STYLED>
__global__ void __launch_bounds__(128, DVG_MINB_BND) k_boundary_eval_batch(const BatchEntry* __restrict__ B,
                                                                           const BSample* samples, const int* order,
                                                                           const int* offsets, int tiles) {
    const int64_t i = (int64_t)(((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 1);
    const bool valid = i < offsets[tiles];
    BSample r{};
    if (valid) r = samples[order[i]];
    const BatchEntry& E = B[valid ? r.scene : 0];
    boundary_eval_pair<STYLED>(E.S, r, valid, E.d_render, E.wsum, E.G);
}

// ------------------------------------------------------------------ background finalisation (background.rs:29-61)
__global__ void k_finalize_background(DevScene S, GradPtrs G) {
    size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (S.bg_image) {
        if (!G.d_background_image || p >= (size_t)S.width * S.height) return;
        const float* im = S.bg_image + 4 * p;
        float* c = G.d_background_image + 4 * p;
        float dr = c[0] * im[3], dg = c[1] * im[3], db = c[2] * im[3];
        float da = c[0] * im[0] + c[1] * im[1] + c[2] * im[2] + c[3];
        c[0] = dr;
        c[1] = dg;
        c[2] = db;
        c[3] = da;
        return;
    }
    if (p != 0) return;
    float* d = G.d_background;
    float r = S.bg[0], g = S.bg[1], b = S.bg[2], a = S.bg[3];
    float nr = d[0] * a, ng = d[1] * a, nb = d[2] * a;
    float na = d[0] * r + d[1] * g + d[2] * b + d[3];
    d[0] = nr;
    d[1] = ng;
    d[2] = nb;
    d[3] = na;
}

// Image::solid / background image copy for scenes without groups (renderer.rs:57-66).
__global__ void k_fill_background(DevScene S, float* out) {
    size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)S.width * S.height) return;
    float4 v = S.bg_image ? reinterpret_cast<const float4*>(S.bg_image)[p]
                          : make_float4(S.bg[0], S.bg[1], S.bg[2], S.bg[3]);
    reinterpret_cast<float4*>(out)[p] = v;
}

// ------------------------------------------------------------------ L2 loss
__global__ void k_l2(const float* img, const float* target, size_t n, float* d_render, float* loss) {
    __shared__ float red[8];
    float s = 0.0f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float d = img[i] - target[i];
        d_render[i] = 2.0f * d;
        s += d * d;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0 && loss) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(loss, t);
    }
}

// ------------------------------------------------------------------ batched per-pixel kernels (grid.y = scene)
__global__ void k_resolve_batch(const BatchEntry* __restrict__ B) {
    const BatchEntry& E = B[blockIdx.y];
    size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)E.S.width * E.S.height) return;
    float r = E.S.bg[0], g = E.S.bg[1], b = E.S.bg[2], a = E.S.bg[3];
    float w = E.wsum[p];
    if (w > 0.0f) {
        float4 c = reinterpret_cast<const float4*>(E.accum)[p];
        r = c.x / w;
        g = c.y / w;
        b = c.z / w;
        a = c.w / w;
    }
    if (a > 1.0e-8f) {
        r = r / a;
        g = g / a;
        b = b / a;
    }
    reinterpret_cast<float4*>(E.image)[p] = make_float4(r, g, b, a);
}
__global__ void k_l2_batch(const BatchEntry* __restrict__ B) {
    __shared__ float red[8];
    const BatchEntry& E = B[blockIdx.y];
    const size_t n = (size_t)E.S.width * E.S.height * 4;
    float s = 0.0f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float d = E.image[i] - E.target[i];
        E.d_render[i] = 2.0f * d;
        s += d * d;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(E.loss, t);
    }
}
__global__ void k_finalize_background_batch(const BatchEntry* __restrict__ B) {
    const BatchEntry& E = B[blockIdx.y];
    size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (E.S.bg_image) {
        if (!E.G.d_background_image || p >= (size_t)E.S.width * E.S.height) return;
        const float* im = E.S.bg_image + 4 * p;
        float* c = E.G.d_background_image + 4 * p;
        float dr = c[0] * im[3], dg = c[1] * im[3], db = c[2] * im[3];
        float da = c[0] * im[0] + c[1] * im[1] + c[2] * im[2] + c[3];
        c[0] = dr;
        c[1] = dg;
        c[2] = db;
        c[3] = da;
        return;
    }
    if (p != 0) return;
    float* d = E.G.d_background;
    float r = E.S.bg[0], g = E.S.bg[1], b = E.S.bg[2], a = E.S.bg[3];
    float nr = d[0] * a, ng = d[1] * a, nb = d[2] * a;
    float na = d[0] * r + d[1] * g + d[2] * b + d[3];
    d[0] = nr;
    d[1] = ng;
    d[2] = nb;
    d[3] = na;
}

}  // namespace dvgb

// ------------------------------------------------------------------ launchers
namespace dvgb {

int launch_binning(const DevScene& S, const float4* g_bbox, int* counts, int* offsets, int* entries,
                   cudaStream_t stream) {
    const int tiles = S.tiles_x * S.tiles_y;
    if (!entries) {
        k_bin_count<<<tiles, 256, 0, stream>>>(S, g_bbox, counts);
        k_bin_scan<<<1, 1024, 0, stream>>>(counts, tiles, offsets);
        return 2;
    }
    k_bin_write<<<tiles, 256, 0, stream>>>(S, g_bbox, offsets, entries);
    return 1;
}
int launch_forward(const DevScene& S, const SampleParams& sp, float* accum, float* wsum, unsigned* status,
                   cudaStream_t stream) {
    const int hw = TILE + 2 * S.filter_ri;
    size_t smem = S.filter_ri <= MAX_SMEM_RI ? (size_t)hw * hw * 5 * sizeof(float) : 0;
    dim3 grid(launch_tiles(S, sp), sp.sxn * sp.syn);
    if (sp.fwd_occ == 2)
        k_forward<2><<<grid, 256, smem, stream>>>(S, sp, accum, wsum, status);
    else if (sp.fwd_occ == 1)
        k_forward<3><<<grid, 256, smem, stream>>>(S, sp, accum, wsum, status);
    else
        k_forward<4><<<grid, 256, smem, stream>>>(S, sp, accum, wsum, status);
    return 1;
}
int launch_weights(const DevScene& S, const SampleParams& sp, float* wsum, cudaStream_t stream) {
    dim3 grid(launch_tiles(S, sp), sp.sxn * sp.syn);
    k_weights<<<grid, 256, 0, stream>>>(S, sp, wsum);
    return 1;
}
int launch_resolve(const DevScene& S, const float* accum, const float* wsum, float* out, cudaStream_t stream) {
    size_t n = (size_t)S.width * S.height;
    k_resolve<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(S, accum, wsum, out);
    return 1;
}
int launch_interior(const DevScene& S, const SampleParams& sp, const float* d_render, const float* wsum,
                    const GradPtrs& G, unsigned* status, cudaStream_t stream) {
    dim3 grid(launch_tiles(S, sp), sp.sxn * sp.syn);
    if (sp.frag) k_interior_cached<<<grid, 256, 0, stream>>>(S, sp, d_render, wsum, G, status);
    k_interior<<<grid, 256, 0, stream>>>(S, sp, d_render, wsum, G, status);
    return sp.frag ? 2 : 1;
}
int launch_boundary(const DevScene& S, const BoundaryParams& bp, const float* d_render, const float* wsum,
                    const GradPtrs& G, BSample* samples, int* key, int* counts, int* order, uint64_t capacity,
                    cudaStream_t stream) {
    const uint64_t n = bp.num_samples;  // samples [bp.sample_base, n)
    const int tiles = S.tiles_x * S.tiles_y * bnd_buckets(bp.cell);  // sort buckets
    int launches = 0;
    for (uint64_t base = bp.sample_base; base < n; base += capacity) {
        const uint64_t cnt = base + capacity < n ? capacity : n - base;
        BoundaryParams b = bp;
        b.sample_base = base;
        b.slot_base = base;
        b.num_samples = base + cnt;
        cudaMemsetAsync(counts, 0, sizeof(int) * (2 * (size_t)tiles + 1), stream);
        k_boundary_gen<<<(unsigned)((cnt + 255) / 256), 256, 0, stream>>>(S, b, samples, key, counts);
        int* offsets = counts + tiles;  // tiles + 1 entries
        launches += launch_scan(counts, tiles, offsets, counts + 2 * (size_t)tiles + 1, stream);
        // reuse the count array as the scatter cursor (a copy of the exclusive offsets)
        cudaMemcpyAsync(counts, offsets, sizeof(int) * (size_t)tiles, cudaMemcpyDeviceToDevice, stream);
        k_boundary_scatter<<<(unsigned)((cnt + 255) / 256), 256, 0, stream>>>(key, cnt, counts, order);
        if (S.styled)
            k_boundary_eval<true><<<(unsigned)((2 * cnt + 127) / 128), 128, 0, stream>>>(S, samples, order, offsets,
                                                                                      tiles, d_render, wsum, G);
        else
            k_boundary_eval<false><<<(unsigned)((2 * cnt + 127) / 128), 128, 0, stream>>>(S, samples, order, offsets,
                                                                                       tiles, d_render, wsum, G);
        launches += 3;
    }
    return launches;
}
int launch_finalize_background(const DevScene& S, const GradPtrs& G, cudaStream_t stream) {
    size_t n = S.bg_image ? (size_t)S.width * S.height : 1;
    k_finalize_background<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(S, G);
    return 1;
}
// Batched step launchers (one launch per stage for all scenes).
// CTAs of a persistent launch: as many as the GPU holds at once (and no more than items).
template <typename K>
int persistent_grid(K kernel, size_t smem, int items) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem);
    return std::max(1, std::min(items, std::max(per_sm, 1) * std::max(sms, 1)));
}
int launch_forward_batch(const BatchEntry* B, const int2* work, int items, int* counter, int max_ri, int occ,
                         cudaStream_t stream) {
    const int hw = TILE + 2 * max_ri;
    size_t smem = max_ri <= MAX_SMEM_RI ? (size_t)hw * hw * 5 * sizeof(float) : 0;
    if (occ == 2) {
        const int grid = counter ? persistent_grid(k_forward_batch<2>, smem, items) : items;
        k_forward_batch<2><<<grid, 256, smem, stream>>>(B, work, items, counter);
    } else if (occ == 1) {
        const int grid = counter ? persistent_grid(k_forward_batch<3>, smem, items) : items;
        k_forward_batch<3><<<grid, 256, smem, stream>>>(B, work, items, counter);
    } else {
        const int grid = counter ? persistent_grid(k_forward_batch<4>, smem, items) : items;
        k_forward_batch<4><<<grid, 256, smem, stream>>>(B, work, items, counter);
    }
    return 1;
}
int launch_pixels_batch(const BatchEntry* B, int nscenes, size_t max_pixels, int which, cudaStream_t stream) {
    if (which == 0) {
        dim3 grid((unsigned)((max_pixels + 255) / 256), nscenes);
        k_resolve_batch<<<grid, 256, 0, stream>>>(B);
    } else if (which == 1) {
        unsigned bx = (unsigned)((max_pixels * 4 + 255) / 256);
        if (bx > 512) bx = 512;
        dim3 grid(bx, nscenes);
        k_l2_batch<<<grid, 256, 0, stream>>>(B);
    } else {
        dim3 grid((unsigned)((max_pixels + 255) / 256), nscenes);
        k_finalize_background_batch<<<grid, 256, 0, stream>>>(B);
    }
    return 1;
}
int launch_interior_batch(const BatchEntry* B, const int2* work, int items, int* counters, unsigned* status,
                          cudaStream_t stream) {
    int* c0 = counters ? counters : nullptr;
    int* c1 = counters ? counters + 1 : nullptr;
    k_interior_cached_batch<<<c0 ? persistent_grid(k_interior_cached_batch, 0, items) : items, 256, 0, stream>>>(
        B, work, items, c0, status);
    k_interior_batch<<<c1 ? persistent_grid(k_interior_batch, 0, items) : items, 256, 0, stream>>>(B, work, items, c1,
                                                                                                  status);
    return 2;
}
int launch_boundary_batch(const BatchEntry* B, int nscenes, uint64_t total, int total_tiles, int cell, bool styled,
                          BSample* samples, int* key, int* counts, int* order, cudaStream_t stream) {
    if (total == 0) return 0;
    total_tiles *= bnd_buckets(cell);  // sort buckets
    cudaMemsetAsync(counts, 0, sizeof(int) * (2 * (size_t)total_tiles + 1), stream);
    k_boundary_gen_batch<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(B, nscenes, total, cell, samples,
                                                                              key, counts);
    int* offsets = counts + total_tiles;
    const int scans = launch_scan(counts, total_tiles, offsets, counts + 2 * (size_t)total_tiles + 1, stream);
    cudaMemcpyAsync(counts, offsets, sizeof(int) * (size_t)total_tiles, cudaMemcpyDeviceToDevice, stream);
    k_boundary_scatter<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(key, total, counts, order);
    if (styled)
        k_boundary_eval_batch<true><<<(unsigned)((2 * total + 127) / 128), 128, 0, stream>>>(B, samples, order,
                                                                                         offsets, total_tiles);
    else
        k_boundary_eval_batch<false><<<(unsigned)((2 * total + 127) / 128), 128, 0, stream>>>(B, samples, order,
                                                                                          offsets, total_tiles);
    return 3 + scans;
}

int launch_fill_background(const DevScene& S, float* out, cudaStream_t stream) {
    size_t n = (size_t)S.width * S.height;
    k_fill_background<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(S, out);
    return 1;
}
int launch_l2(const float* img, const float* target, size_t n, float* d_render, float* loss, cudaStream_t stream) {
    unsigned blocks = (unsigned)((n + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    if (blocks == 0) blocks = 1;
    k_l2<<<blocks, 256, 0, stream>>>(img, target, n, d_render, loss);
    return 1;
}

}  // namespace dvgb
