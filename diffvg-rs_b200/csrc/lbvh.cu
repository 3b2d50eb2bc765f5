// lbvh.cu — linear BVH (Karras 2012, "Maximizing Parallelism in the Construction of
// BVHs, Octrees, and k-d Trees") over axis-aligned boxes, built entirely on the GPU:
//   1. 32-bit Morton code of each box centre (16 bits per axis, normalised to the
//      bounds of the centres), key = code << 32 | box index (unique keys);
//   2. bitonic sort of the keys (unique keys: any correct sort gives one order);
//   3. topology: every internal node finds its key range and split from the common
//      prefix lengths of its neighbours' keys, independently of the others;
//   4. bounds bottom-up: the second child to arrive at a parent unions both.
// Every step is integer work or exact min / max, and the codes use f32 arithmetic
// without contraction, so the tree is bit-for-bit the one a CPU build of the same
// steps produces (the oracle's lbvh build; tests/test_lbvh.py).
//
// Layout: internal nodes 0 .. n-2 (root 0), leaves n-1 .. 2n-2 in sorted order;
// children[i] = (left, right) node ids; leaf k holds box key[k] & 0xffffffff.
// Exposed through dvg_lbvh_build.  The scene's own BVHs stay the crate's median
// splits (its closest-point search breaks distance ties by traversal order), and
// its closest-group search keeps the crate's group order (see prefilter.cu).
#include "kernels.cuh"

namespace dvgb {
namespace {

__device__ __forceinline__ uint32_t spread16(uint32_t v) {  // 16 bits -> even bit positions
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
__device__ __forceinline__ uint32_t quantise(float c, float lo, float ext) {
    float u = ext > 0.0f ? (c - lo) / ext : 0.0f;
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    const float s = u * 65536.0f;
    return s >= 65535.0f ? 65535u : (uint32_t)s;
}

// Bounds of the box centres (single CTA; boxes are few compared with samples).
__global__ void __launch_bounds__(1024) k_lbvh_extent(const float4* boxes, int n, float4* ext) {
    __shared__ float s[4][32];
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 b = boxes[i];
        const float cx = (b.x + b.z) * 0.5f, cy = (b.y + b.w) * 0.5f;
        x0 = fminf(x0, cx);
        y0 = fminf(y0, cy);
        x1 = fmaxf(x1, cx);
        y1 = fmaxf(y1, cy);
    }
    for (int o = 16; o > 0; o >>= 1) {
        x0 = fminf(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        y0 = fminf(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        x1 = fmaxf(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        y1 = fmaxf(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        s[0][wid] = x0;
        s[1][wid] = y0;
        s[2][wid] = x1;
        s[3][wid] = y1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) / 32;
        float a = s[0][0], b = s[1][0], c = s[2][0], d = s[3][0];
        for (int w = 1; w < nw; ++w) {
            a = fminf(a, s[0][w]);
            b = fminf(b, s[1][w]);
            c = fmaxf(c, s[2][w]);
            d = fmaxf(d, s[3][w]);
        }
        *ext = make_float4(a, b, c, d);
    }
}

__global__ void k_lbvh_keys(const float4* boxes, int n, int padded, const float4* ext, uint64_t* keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= padded) return;
    if (i >= n) {
        keys[i] = ~0ull;
        return;
    }
    const float4 e = *ext;
    const float4 b = boxes[i];
    const float cx = (b.x + b.z) * 0.5f, cy = (b.y + b.w) * 0.5f;
    const uint32_t qx = quantise(cx, e.x, e.z - e.x), qy = quantise(cy, e.y, e.w - e.y);
    const uint32_t code = spread16(qx) | (spread16(qy) << 1);
    keys[i] = ((uint64_t)code << 32) | (uint32_t)i;
}

// One compare-exchange stage of a bitonic sort over `padded` (a power of two) keys.
__global__ void k_bitonic_stage(uint64_t* keys, int padded, int k, int j) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= padded) return;
    const int l = i ^ j;
    if (l <= i) return;
    const uint64_t a = keys[i], b = keys[l];
    const bool ascending = (i & k) == 0;
    if (ascending ? a > b : a < b) {
        keys[i] = b;
        keys[l] = a;
    }
}
// All stages with j < 1024 of one k run inside a CTA of 1024 keys in shared memory.
__global__ void __launch_bounds__(1024) k_bitonic_local(uint64_t* keys, int padded, int k, int jmax) {
    __shared__ uint64_t s[1024];
    const int base = blockIdx.x * 1024;
    const int t = threadIdx.x;
    if (base + t < padded) s[t] = keys[base + t];
    __syncthreads();
    for (int j = jmax; j > 0; j >>= 1) {
        const int i = base + t, l = i ^ j;
        if (l > i && l < padded) {
            const uint64_t a = s[t], b = s[l - base];
            const bool ascending = (i & k) == 0;
            if (ascending ? a > b : a < b) {
                s[t] = b;
                s[l - base] = a;
            }
        }
        __syncthreads();
    }
    if (base + t < padded) keys[base + t] = s[t];
}

__device__ __forceinline__ int prefix(const uint64_t* keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(keys[i] ^ keys[j]);
}
__global__ void k_lbvh_topology(const uint64_t* keys, int n, int2* children, int* parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = prefix(keys, n, i, i + 1) - prefix(keys, n, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = prefix(keys, n, i, i - d);
    int lmax = 2;
    while (prefix(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (prefix(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = prefix(keys, n, i, j);
    int s = 0;
    for (int div = 2;; div *= 2) {
        const int t = (l + div - 1) / div;
        if (prefix(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int gamma = i + s * d + (d < 0 ? -1 : 0);
    const int left = (i < j ? i : j) == gamma ? (n - 1) + gamma : gamma;
    const int right = (i > j ? i : j) == gamma + 1 ? (n - 1) + gamma + 1 : gamma + 1;
    children[i] = make_int2(left, right);
    parent[left] = i;
    parent[right] = i;
}
__global__ void k_lbvh_bounds(const float4* boxes, const uint64_t* keys, int n, const int* item_map,
                              const int2* children, const int* parent, int* flags, float4* bounds, int* leaf_item) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int item = (int)(keys[k] & 0xffffffffu);
    leaf_item[k] = item_map ? item_map[item] : item;
    int node = (n - 1) + k;
    bounds[node] = boxes[item];
    if (n == 1) return;
    __threadfence();
    node = parent[node];
    while (true) {
        if (atomicAdd(&flags[node], 1) == 0) return;  // the sibling subtree is not done yet
        __threadfence();
        const int2 c = children[node];
        const float4 a = __ldcg(&bounds[c.x]), b = __ldcg(&bounds[c.y]);
        bounds[node] = make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
        __threadfence();
        if (node == 0) return;
        node = parent[node];
    }
}

}  // namespace

int lbvh_padded(int n) {
    int p = 1;
    while (p < n) p *= 2;
    return p;
}

int launch_lbvh_build(const float4* boxes, int n, const int* item_map, LbvhBufs& L, cudaStream_t stream) {
    if (n <= 0) return 0;
    const int padded = lbvh_padded(n);
    int launches = 0;
    k_lbvh_extent<<<1, 1024, 0, stream>>>(boxes, n, L.extent);
    k_lbvh_keys<<<(padded + 255) / 256, 256, 0, stream>>>(boxes, n, padded, L.extent, L.keys);
    launches += 2;
    for (int k = 2; k <= padded; k *= 2) {
        int j = k / 2;
        for (; j >= 1024; j /= 2) {
            k_bitonic_stage<<<(padded + 255) / 256, 256, 0, stream>>>(L.keys, padded, k, j);
            ++launches;
        }
        k_bitonic_local<<<(padded + 1023) / 1024, 1024, 0, stream>>>(L.keys, padded, k, j);
        ++launches;
    }
    if (n > 1) {
        cudaMemsetAsync(L.flags, 0, sizeof(int) * (size_t)(n - 1), stream);
        k_lbvh_topology<<<(n - 1 + 255) / 256, 256, 0, stream>>>(L.keys, n, L.children, L.parent);
        ++launches;
    }
    k_lbvh_bounds<<<(n + 255) / 256, 256, 0, stream>>>(boxes, L.keys, n, item_map, L.children, L.parent, L.flags,
                                                      L.bounds, L.leaf_item);
    return launches + 1;
}


}  // namespace dvgb
