// refit.cu — the on-device optimisation step of a batch: Adam on path points (and
// optionally paint parameters), then the scene tables derived from the points are
// rebuilt in place, so the next step renders the updated scene with no host
// preparation and no host round trip (the whole step stays inside one CUDA graph).
//
// The rebuild repeats the host preparation (prepare.cpp) operation for operation,
// in f32 without contraction (and f64 for the canvas boxes), so a re-prepared scene
// holds bit-for-bit the tables a fresh upload of the same points would get:
//   segments          src/distance/bvh.rs:255-364 (control points, closed-path wrap)
//   path / group BVH  src/distance/bvh.rs:156-238 (median split on the longest axis,
//                     leaf <= 8, stable sort by box centre) — the node layout depends
//                     only on the element counts, so only bounds and leaf order change
//   shape bounds      src/distance/shape.rs:9-78 (transformed points, stroke padding)
//   boundary tables   src/backward/boundary.rs:200-451 (lengths, CDFs, PMFs)
#include "kernels.cuh"

namespace dvgb {
namespace {

constexpr int kLeaf = 8;  // BVH_LEAF_SIZE, src/distance/bvh.rs:12
constexpr int kStack = 64;

struct RBox {
    float x0, y0, x1, y1;
};
__device__ __forceinline__ RBox rbox_empty() { return RBox{INFINITY, INFINITY, -INFINITY, -INFINITY}; }
__device__ __forceinline__ void rbox_grow(RBox& b, const RBox& o) {
    b.x0 = fminf(b.x0, o.x0);
    b.y0 = fminf(b.y0, o.y0);
    b.x1 = fmaxf(b.x1, o.x1);
    b.y1 = fmaxf(b.y1, o.y1);
}
__device__ __forceinline__ void rbox_grow_pt(RBox& b, float x, float y) {
    b.x0 = fminf(b.x0, x);
    b.y0 = fminf(b.y0, y);
    b.x1 = fmaxf(b.x1, x);
    b.y1 = fmaxf(b.y1, y);
}
__device__ __forceinline__ RBox rbox_inflate(RBox b, float pad) {  // src/distance/shape.rs:92-99
    pad = fmaxf(pad, 0.0f);
    return RBox{b.x0 - pad, b.y0 - pad, b.x1 + pad, b.y1 + pad};
}
__device__ __forceinline__ RBox from4(float4 v) { return RBox{v.x, v.y, v.z, v.w}; }
__device__ __forceinline__ float4 to4(const RBox& b) { return make_float4(b.x0, b.y0, b.x1, b.y1); }

// Padded bounds of one segment from its (already rebuilt) control points and radii.
__device__ __forceinline__ RBox seg_box(const DevScene& S, int sid) {
    const float4 a = S.seg_p[2 * sid], b = S.seg_p[2 * sid + 1], r = S.seg_r[sid];
    RBox bb = rbox_empty();
    rbox_grow_pt(bb, a.x, a.y);
    rbox_grow_pt(bb, a.z, a.w);
    rbox_grow_pt(bb, b.x, b.y);
    rbox_grow_pt(bb, b.z, b.w);
    const float rmax = fmaxf(fmaxf(r.x, r.y), fmaxf(r.z, r.w));
    return rbox_inflate(bb, rmax);
}

// Stable bottom-up merge sort of ids[0..n) by keys (ascending; equal keys keep
// their order, as the stable sort of the host build).  tmp_ids / tmp_keys: n each.
__device__ void stable_sort(int* ids, float* keys, int* tmp_ids, float* tmp_keys, int n) {
    int* si = ids;
    float* sk = keys;
    int* di = tmp_ids;
    float* dk = tmp_keys;
    for (int w = 1; w < n; w *= 2) {
        for (int lo = 0; lo < n; lo += 2 * w) {
            const int mid = min(lo + w, n), hi = min(lo + 2 * w, n);
            int i = lo, j = mid;
            for (int k = lo; k < hi; ++k) {
                const bool take_right = j < hi && (i >= mid || sk[j] < sk[i]);
                if (take_right) {
                    di[k] = si[j];
                    dk[k] = sk[j];
                    ++j;
                } else {
                    di[k] = si[i];
                    dk[k] = sk[i];
                    ++i;
                }
            }
        }
        int* ti = si;
        si = di;
        di = ti;
        float* tk = sk;
        sk = dk;
        dk = tk;
    }
    if (si != ids)
        for (int k = 0; k < n; ++k) {
            ids[k] = si[k];
            keys[k] = sk[k];
        }
}

// Rebuilds one median-split BVH in place.  leaf[0..n) holds the element ids in
// their original order on entry and the leaf order on exit; node ids, skip links,
// right-child links and leaf ranges are read from the existing meta (they depend
// only on n).  Returns false when the stored layout does not match the recursion.
template <typename BoxOf>
__device__ bool rebuild_bvh(int* leaf, int leaf_base, int n, int node_off, int node_cnt, float4* bounds,
                            const int4* meta, int* scratch_ids, float* scratch_keys, BoxOf box_of) {
    int st_lo[kStack], st_hi[kStack], st_node[kStack];
    int top = 0;
    st_lo[0] = 0;
    st_hi[0] = n;
    st_node[0] = node_off;
    top = 1;
    while (top > 0) {
        --top;
        const int lo = st_lo[top], hi = st_hi[top], node = st_node[top];
        if (node < node_off || node >= node_off + node_cnt) return false;
        const int4 m = meta[node];
        if (m.y != leaf_base + lo) return false;
        RBox b = rbox_empty();
        for (int i = lo; i < hi; ++i) rbox_grow(b, box_of(leaf[i]));
        bounds[node] = to4(b);
        const int cnt = hi - lo;
        if (cnt <= kLeaf) {
            if (m.z != cnt) return false;
            continue;
        }
        if (m.z != 0 || m.w < 0 || top + 2 > kStack) return false;
        const int axis = (b.x1 - b.x0) >= (b.y1 - b.y0) ? 0 : 1;
        int* ids = scratch_ids;
        float* keys = scratch_keys;
        for (int i = 0; i < cnt; ++i) {
            const int id = leaf[lo + i];
            const RBox e = box_of(id);
            ids[i] = id;
            keys[i] = axis == 0 ? (e.x0 + e.x1) * 0.5f : (e.y0 + e.y1) * 0.5f;
        }
        stable_sort(ids, keys, ids + cnt, keys + cnt, cnt);
        for (int i = 0; i < cnt; ++i) leaf[lo + i] = ids[i];
        const int mid = lo + cnt / 2;
        st_lo[top] = mid;  // right subtree (popped second)
        st_hi[top] = hi;
        st_node[top] = m.w;
        ++top;
        st_lo[top] = lo;  // left subtree = next node in preorder
        st_hi[top] = mid;
        st_node[top] = node + 1;
        ++top;
    }
    return true;
}

__device__ __forceinline__ float2 path_pt(const DevScene& S, int po, int pc, bool closed, int index) {
    const int i = closed ? index % pc : index;  // src/path_utils.rs:7-16
    return S.points[po + i];
}
__device__ __forceinline__ float seg_chord(float x0, float y0, float x1, float y1) {
    const float dx = x1 - x0, dy = y1 - y0;
    return sqrtf(dx * dx + dy * dy);
}
// Polyline length of one segment (src/backward/boundary.rs:230-309); *ok = false
// when a control point is missing (open path running past its last point).
__device__ float seg_length(const DevScene& S, int po, int pc, bool closed, int pid, int nc, bool* ok) {
    float q[8];
    const int np = nc + 2;
    *ok = true;
    for (int k = 0; k < np; ++k) {
        if (pc == 0 || (!closed && pid + k >= pc)) {
            *ok = false;
            return 0.0f;
        }
        const float2 p = path_pt(S, po, pc, closed, pid + k);
        q[2 * k] = p.x;
        q[2 * k + 1] = p.y;
    }
    if (nc == 0) return seg_chord(q[0], q[1], q[2], q[3]);
    if (nc == 1) {
        const float t = 0.5f, tt = 1.0f - t;
        const float vx = q[0] * (tt * tt) + q[2] * (2.0f * tt * t) + q[4] * (t * t);
        const float vy = q[1] * (tt * tt) + q[3] * (2.0f * tt * t) + q[5] * (t * t);
        return seg_chord(q[0], q[1], vx, vy) + seg_chord(vx, vy, q[4], q[5]);
    }
    float v[4];
    for (int k = 0; k < 2; ++k) {
        const float t = k == 0 ? 1.0f / 3.0f : 2.0f / 3.0f, tt = 1.0f - t;
        v[2 * k] = q[0] * (tt * tt * tt) + q[2] * (3.0f * tt * tt * t) + q[4] * (3.0f * tt * t * t) +
                   q[6] * (t * t * t);
        v[2 * k + 1] = q[1] * (tt * tt * tt) + q[3] * (3.0f * tt * tt * t) + q[5] * (3.0f * tt * t * t) +
                       q[7] * (t * t * t);
    }
    return seg_chord(q[0], q[1], v[0], v[1]) + seg_chord(v[0], v[1], v[2], v[3]) + seg_chord(v[2], v[3], q[6], q[7]);
}

// Adam (PyTorch's default form: no weight decay, no AMSGrad) on every selected
// parameter of every scene; thread = parameter, grid.y = scene.
__global__ void k_adam_batch(BatchEntry* B, const RefitEntry* R, AdamParams ap, const int* step) {
    const int scene = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const RefitEntry& r = R[scene];
    const BatchEntry& e = B[scene];
    const int np = ap.points ? 2 * r.n_points : 0;
    const int nq = ap.paints ? 4 * r.n_paints : 0;
    if (i >= np + nq) return;
    const float t = (float)(*step + 1);
    const float bc1 = 1.0f - powf(ap.beta1, t), bc2 = 1.0f - powf(ap.beta2, t);
    const float step_size = ap.lr / bc1, bc2_sqrt = sqrtf(bc2);
    float *p, *m, *v;
    float g;
    if (i < np) {
        p = reinterpret_cast<float*>(const_cast<float2*>(e.S.points)) + i;
        m = r.m_points + i;
        v = r.v_points + i;
        g = e.G.d_points[i];
    } else {
        const int j = i - np;
        p = reinterpret_cast<float*>(const_cast<float4*>(e.S.paint_params)) + j;
        m = r.m_paints + j;
        v = r.v_paints + j;
        g = e.G.d_paint_params[j];
    }
    const float mn = ap.beta1 * *m + (1.0f - ap.beta1) * g;
    const float vn = ap.beta2 * *v + (1.0f - ap.beta2) * (g * g);
    *m = mn;
    *v = vn;
    const float denom = sqrtf(vn) / bc2_sqrt + ap.eps;
    *p = *p - step_size * (mn / denom);
}
__global__ void k_step_inc(int* step) { *step += 1; }

// Thread = path: control points -> segments, path BVH, path length and segment
// CDF, and the path shape's padded group-space bounds.
__global__ void k_refit_paths(BatchEntry* B, const RefitEntry* R, unsigned* status) {
    const int scene = blockIdx.y;
    const int path = blockIdx.x * blockDim.x + threadIdx.x;
    const DevScene& S = B[scene].S;
    const RefitEntry& r = R[scene];
    if (path >= S.num_paths) return;
    const int4 pi = S.p_info[2 * path], pi2 = S.p_info[2 * path + 1];
    const int seg_off = pi.x, nseg = pi.y, node_off = pi.z, node_cnt = pi.w;
    const int po = pi2.x, pc = pi2.y, co = pi2.z, flags = pi2.w;
    const bool closed = flags & PF_CLOSED, thick = flags & PF_THICK;
    const int shape = S.p_shape[path];

    // segments (src/distance/bvh.rs:255-364)
    float4* seg_p = const_cast<float4*>(S.seg_p);
    for (int k = 0; k < nseg; ++k) {
        const int4 sm = S.seg_meta[seg_off + k];
        const int np = sm.x + 2, pid = sm.z;
        float q[8];
        for (int j = 0; j < np; ++j) {
            const float2 p = path_pt(S, po, pc, closed, pid + j);
            q[2 * j] = p.x;
            q[2 * j + 1] = p.y;
        }
        for (int j = np; j < 4; ++j) {
            q[2 * j] = q[2 * (np - 1)];
            q[2 * j + 1] = q[2 * (np - 1) + 1];
        }
        seg_p[2 * (seg_off + k)] = make_float4(q[0], q[1], q[2], q[3]);
        seg_p[2 * (seg_off + k) + 1] = make_float4(q[4], q[5], q[6], q[7]);
    }

    // path BVH
    if (node_cnt > 0) {
        int* leaf = const_cast<int*>(S.pl_segs) + S.pn_meta[node_off].y;
        for (int k = 0; k < nseg; ++k) leaf[k] = seg_off + k;
        const bool ok = rebuild_bvh(leaf, S.pn_meta[node_off].y, nseg, node_off, node_cnt,
                                    const_cast<float4*>(S.pn_bounds),
                                    S.pn_meta, r.sort_ids + 2 * seg_off, r.sort_keys + 2 * seg_off,
                                    [&](int sid) { return seg_box(S, sid); });
        if (!ok) atomicOr(status, ST_REFIT_LAYOUT);
    }

    // path length (src/backward/boundary.rs:200-309) and segment CDF (:349-451)
    const int cc = S.path_cdf_info[shape].y;
    float l = 0.0f;
    if (pc > 0) {
        int pid = 0;
        for (int k = 0; k < cc; ++k) {
            const int nc = S.ncp[co + k];
            if (nc > 2) break;
            bool ok;
            const float sl = seg_length(S, po, pc, closed, pid, nc, &ok);
            if (!ok) break;
            l += sl;
            pid += nc + 1;
        }
    }
    const_cast<float*>(S.shape_len)[shape] = l;
    if (cc > 0) {
        int4* info = const_cast<int4*>(S.path_cdf_info) + shape;
        const bool valid = l > 0.0f && isfinite(l);
        const float inv_length = valid ? 1.0f / l : 0.0f;
        float* pmf = const_cast<float*>(S.path_pmf) + info->x;
        float* cdf = const_cast<float*>(S.path_cdf) + info->x;
        int pid = 0;
        float prev = 0.0f;
        for (int k = 0; k < cc; ++k) {
            const int nc = S.ncp[co + k];
            float sl = 0.0f;
            if (nc <= 2) {
                bool ok;
                sl = seg_length(S, po, pc, closed, pid, nc, &ok);
                if (!ok) sl = 0.0f;
                pid += nc + 1;
            }
            const float sn = sl * inv_length;
            pmf[k] = sn;
            const float acc = sn + (k == 0 ? 0.0f : prev);
            cdf[k] = acc;
            prev = acc;
        }
        info->z = valid ? 1 : 0;
        const_cast<float*>(S.path_len)[shape] = valid ? l : 0.0f;
    }

    // padded group-space bounds of the path shape (src/distance/shape.rs:9-78)
    if (pc > 0) {
        const float* t = S.s_xform + 9 * shape;
        const bool ident = S.s_info[shape].y & SF_IDENTITY;
        RBox gb = rbox_empty();
        for (int k = 0; k < pc; ++k) {
            float x = S.points[po + k].x, y = S.points[po + k].y;
            if (!ident) {
                const float ox = t[0] * x + t[1] * y + t[2];
                const float oy = t[3] * x + t[4] * y + t[5];
                x = ox;
                y = oy;
            }
            rbox_grow_pt(gb, x, y);
        }
        const float sx = sqrtf(t[0] * t[0] + t[3] * t[3]), sy = sqrtf(t[1] * t[1] + t[4] * t[4]);
        const float scale = fmaxf(fmaxf(sx, sy), 0.0f);
        float rad = fabsf(S.s_stroke[shape]) * scale;
        if (thick) {
            float mt = 0.0f;
            for (int k = 0; k < pc; ++k) mt = fmaxf(mt, fabsf(S.thickness[po + k]));
            rad = fmaxf(rad, mt * scale);
        }
        if (rad > 0.0f) rad *= S.s_padmul[shape];
        const_cast<float4*>(S.s_box)[shape] = to4(rbox_inflate(gb, rad));
    }
}

// Thread = group: group BVH over its shapes' padded bounds and the conservative
// canvas-space box used by tile binning.
__global__ void k_refit_groups(BatchEntry* B, const RefitEntry* R, unsigned* status) {
    const int scene = blockIdx.y;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const DevScene& S = B[scene].S;
    const RefitEntry& r = R[scene];
    if (g >= S.num_groups) return;
    const int4 gb = S.g_bvh[g];
    const int node_off = gb.x, node_cnt = gb.y, list_off = gb.z, list_cnt = gb.w;
    if (node_cnt == 0) return;
    const int leaf_base = S.gn_meta[node_off].y;
    int* leaf = const_cast<int*>(S.gl_shapes) + leaf_base;
    int n = 0;
    for (int k = 0; k < list_cnt; ++k) {
        const int sid = S.g_shape_list[list_off + k];
        if (S.s_info[sid].y & SF_HAS_BOUNDS) leaf[n++] = sid;
    }
    const bool ok = rebuild_bvh(leaf, leaf_base, n, node_off, node_cnt, const_cast<float4*>(S.gn_bounds), S.gn_meta,
                                r.sort_ids + 2 * list_off, r.sort_keys + 2 * list_off,
                                [&](int sid) { return from4(S.s_box[sid]); });
    if (!ok) atomicOr(status, ST_REFIT_LAYOUT);
    // canvas-space box of the root (as prepare.cpp, in f64)
    const float4 root = S.gn_bounds[node_off];
    float4* out = r.g_bbox + g;
    const float* c = S.g_c2s + 9 * g;
    const double a = c[0], b = c[1], cc = c[3], dd = c[4], tx = c[2], ty = c[5];
    const double det = a * dd - b * cc;
    const bool finite_root = isfinite(root.x) && isfinite(root.y) && isfinite(root.z) && isfinite(root.w);
    if (fabs(det) < 1e-12 || !finite_root) {
        *out = make_float4(-INFINITY, -INFINITY, INFINITY, INFINITY);
        return;
    }
    const double xs[4] = {root.x, root.z, root.z, root.x}, ys[4] = {root.y, root.y, root.w, root.w};
    double mnx = 1e300, mny = 1e300, mxx = -1e300, mxy = -1e300;
    for (int k = 0; k < 4; ++k) {
        const double lx = xs[k] - tx, ly = ys[k] - ty;
        const double X = (dd * lx - b * ly) / det, Y = (-cc * lx + a * ly) / det;
        mnx = fmin(mnx, X);
        mny = fmin(mny, Y);
        mxx = fmax(mxx, X);
        mxy = fmax(mxy, Y);
    }
    const double pad = 0.5 + 1e-4 * (fabs(mnx) + fabs(mny) + fabs(mxx) + fabs(mxy));
    *out = make_float4((float)(mnx - pad), (float)(mny - pad), (float)(mxx + pad), (float)(mxy + pad));
}

// One thread per scene: the (group, shape) length CDF in group order
// (src/backward/boundary.rs:312-346) and the scene's boundary_ok flag.
__global__ void k_refit_cdf(BatchEntry* B, int nscenes) {
    const int scene = blockIdx.x * blockDim.x + threadIdx.x;
    if (scene >= nscenes) return;
    DevScene& S = B[scene].S;
    const int n = S.bcdf_n;
    float* cdf = const_cast<float*>(S.bcdf);
    float* pmf = const_cast<float*>(S.bpmf);
    float accum = 0.0f;
    for (int k = 0; k < n; ++k) {
        const float l = S.shape_len[S.b_shape[k]];
        accum += l;
        cdf[k] = accum;
        pmf[k] = l;
    }
    const bool ok = S.num_groups > 0 && accum > 0.0f && isfinite(accum) && n > 0;
    if (ok)
        for (int k = 0; k < n; ++k) {
            cdf[k] /= accum;
            pmf[k] /= accum;
        }
    S.boundary_ok = ok ? 1 : 0;
}

}  // namespace

int launch_adam_batch(BatchEntry* B, const RefitEntry* R, int nscenes, int max_params, const AdamParams& ap,
                      int* step, cudaStream_t stream) {
    if (nscenes <= 0 || max_params <= 0) return 0;
    dim3 grid((unsigned)((max_params + 255) / 256), (unsigned)nscenes);
    k_adam_batch<<<grid, 256, 0, stream>>>(B, R, ap, step);
    k_step_inc<<<1, 1, 0, stream>>>(step);
    return 2;
}

int launch_refit_batch(BatchEntry* B, const RefitEntry* R, int nscenes, int max_paths, int max_groups,
                       unsigned* status, cudaStream_t stream) {
    int n = 0;
    if (nscenes <= 0) return 0;
    if (max_paths > 0) {
        k_refit_paths<<<dim3((unsigned)((max_paths + 63) / 64), (unsigned)nscenes), 64, 0, stream>>>(B, R, status);
        ++n;
    }
    if (max_groups > 0) {
        k_refit_groups<<<dim3((unsigned)((max_groups + 63) / 64), (unsigned)nscenes), 64, 0, stream>>>(B, R,
                                                                                                         status);
        ++n;
    }
    k_refit_cdf<<<(unsigned)((nscenes + 31) / 32), 32, 0, stream>>>(B, nscenes);
    return n + 1;
}

}  // namespace dvgb
