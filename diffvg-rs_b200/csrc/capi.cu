// capi.cu — the extern "C" boundary (include/dvg.h) over the sm_100a kernels.
//
// A context owns one CUDA stream, a device status word and grow-only scratch
// buffers; a scene owns one device arena holding every table of the prepared
// scene plus its tile lists and a gradient arena sized for it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dvg.h"
#include "kernels.cuh"
#include "prepare.hpp"

static_assert((int)dvgb::PATH_STYLED == (int)dvgb::PF_STYLED && (int)dvgb::PATH_JOIN_SHIFT == (int)dvgb::PF_JOIN_SHIFT &&
                  (int)dvgb::PATH_CAP_SHIFT == (int)dvgb::PF_CAP_SHIFT,
              "path style bits differ between host preparation and the kernels");
static_assert((int)DVG_JOIN_MITER == (int)dvgb::JOIN_MITER && (int)DVG_JOIN_BEVEL == (int)dvgb::JOIN_BEVEL &&
                  (int)DVG_JOIN_ROUND == (int)dvgb::JOIN_ROUND && (int)DVG_CAP_BUTT == (int)dvgb::CAP_BUTT &&
                  (int)DVG_CAP_SQUARE == (int)dvgb::CAP_SQUARE && (int)DVG_CAP_ROUND == (int)dvgb::CAP_ROUND,
              "join / cap codes differ between the ABI and the kernels");

using namespace dvgb;

namespace {

thread_local std::string g_last_error;

dvg_status fail(dvg_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}
dvg_status cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? DVG_ERR_OUT_OF_MEMORY : DVG_ERR_LAUNCH;
}
#define CK(call)                                           \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    ~DevBuf() {
        if (ptr) cudaFree(ptr);
    }
    cudaError_t reserve(size_t n) {
        if (n <= bytes) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&ptr, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
};

// Packs several host arrays into one blob with 256-byte aligned offsets.
struct Blob {
    std::vector<char> data;
    template <typename T>
    size_t add(const std::vector<T>& v) {
        size_t off = (data.size() + 255) & ~(size_t)255;
        data.resize(off + std::max<size_t>(v.size() * sizeof(T), 16));
        if (!v.empty()) std::memcpy(data.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
};

}  // namespace

struct ProfEvent {
    const char* name;
    cudaEvent_t a, b;
};
struct ProfStat {
    const char* name;
    double ms;
    uint64_t count;
};

struct dvg_context {
    int device = 0;
    bool profiling = false;
    std::vector<ProfEvent> pending;
    std::vector<ProfStat> stats;
    cudaStream_t stream = nullptr;
    unsigned* status = nullptr;  // device word
    DevBuf accum, wsum, image, d_render, target, loss, bg_grad, trans_grad;
    DevBuf bsamples, bkey, border, bcounts;  // boundary-pass scratch
    DevBuf sdf, positions, dvalues;          // signed-distance host calls
    DevBuf frag;                             // fragment cache of the fused calls
    uint64_t launches = 0;
    // Retained render: dvg_render keeps its prepared scene, and its weight image and
    // fragment cache stay valid until the next call that writes them (gen counts
    // those calls), so a dvg_render_backward of the same description and options
    // reuses all three instead of preparing, uploading and re-testing again.
    bool retain = true;
    uint64_t gen = 0;
    dvg_scene* kept = nullptr;
    std::vector<char> kept_key;
    dvg_render_options kept_opts{};
    uint64_t kept_gen = 0;
    bool kept_weights = false, kept_frag = false;
    // The last dvg_shard_forward (its fragment codes serve the shard backward that follows).
    const dvg_scene* shard_scene = nullptr;
    dvg_render_options shard_opts{};
    uint32_t shard_t0 = 0, shard_t1 = 0;
    uint64_t shard_gen = 0;
    bool shard_frag = false;
    dvg_tuning shard_tune{};  // the scene's launch shape when its fragment codes were written
};

struct dvg_scene {
    dvg_context* ctx = nullptr;
    HostScene host;
    DevScene dev{};
    DevBuf arena;
    DevBuf tiles;    // counts, offsets
    DevBuf entries;  // tile entries
    DevBuf grads;    // gradient arena (device)
    size_t grad_off[11] = {0};
    size_t grad_floats = 0;
    size_t arena_bytes = 0;  // bytes of prepared tables in `arena`
    const float4* g_bbox = nullptr;
    dvg_tuning tune{1, 4, 16, 0, 0};  // launch shape (dvg_scene_set_tuning / dvg_scene_autotune)
};

namespace {

// Offsets of each gradient part inside the scene's gradient arena (in floats).
void layout_grads(dvg_scene* sc) {
    const HostScene& h = sc->host;
    size_t sizes[11] = {4 * (size_t)h.num_shapes, 9 * (size_t)h.num_shapes, h.num_shapes, 2 * (size_t)h.total_points,
                        h.total_points,           9 * (size_t)h.num_groups, 4 * (size_t)h.num_paints,
                        h.total_stops,            4 * (size_t)h.total_stops, 1, 4};
    size_t off = 0;
    for (int i = 0; i < 11; ++i) {
        sc->grad_off[i] = off;
        off += (sizes[i] + 63) & ~(size_t)63;
    }
    sc->grad_floats = off;
}
GradPtrs device_grads(dvg_scene* sc) {
    float* b = sc->grads.as<float>();
    GradPtrs g;
    g.d_shape_params = b + sc->grad_off[0];
    g.d_shape_transform = b + sc->grad_off[1];
    g.d_shape_stroke_width = b + sc->grad_off[2];
    g.d_points = b + sc->grad_off[3];
    g.d_thickness = b + sc->grad_off[4];
    g.d_group_transform = b + sc->grad_off[5];
    g.d_paint_params = b + sc->grad_off[6];
    g.d_stop_offsets = b + sc->grad_off[7];
    g.d_stop_colors = b + sc->grad_off[8];
    g.d_filter_radius = b + sc->grad_off[9];
    g.d_background = b + sc->grad_off[10];
    g.d_background_image = nullptr;
    g.d_translation = nullptr;
    return g;
}

// Byte image of a scene description: every scalar and every array it points to
// (a marker byte for each optional array left NULL).  Equal images prepare to the
// same device scene.
void desc_key(const dvg_scene_desc* d, std::vector<char>& k) {
    k.clear();
    auto put = [&](const void* p, size_t n) {
        const char* c = static_cast<const char*>(p);
        k.insert(k.end(), c, c + n);
    };
    auto arr = [&](const void* p, size_t n) {
        const char mark = p ? 1 : 0;
        put(&mark, 1);
        if (p && n) put(p, n);
    };
    const size_t ns = d->num_shapes, ng = d->num_groups, np = d->num_paints;
    put(&d->width, sizeof d->width);
    put(&d->height, sizeof d->height);
    put(d->background, sizeof d->background);
    put(&d->filter_type, sizeof d->filter_type);
    put(&d->filter_radius, sizeof d->filter_radius);
    put(&d->num_shapes, sizeof d->num_shapes);
    put(&d->total_ctrl, sizeof d->total_ctrl);
    put(&d->total_points, sizeof d->total_points);
    put(&d->num_groups, sizeof d->num_groups);
    put(&d->total_group_shapes, sizeof d->total_group_shapes);
    put(&d->num_paints, sizeof d->num_paints);
    put(&d->total_stops, sizeof d->total_stops);
    arr(d->background_image, d->background_image ? (size_t)d->width * d->height * 4 * sizeof(float) : 0);
    arr(d->shape_kind, ns * 4);
    arr(d->shape_params, ns * 16);
    arr(d->shape_transform, ns * 36);
    arr(d->shape_stroke_width, ns * 4);
    arr(d->shape_stroke_join, ns * 4);
    arr(d->shape_stroke_cap, ns * 4);
    arr(d->shape_miter_limit, ns * 4);
    arr(d->path_ctrl_offset, ns * 4);
    arr(d->path_ctrl_count, ns * 4);
    arr(d->path_point_offset, ns * 4);
    arr(d->path_point_count, ns * 4);
    arr(d->path_flags, ns * 4);
    arr(d->num_control_points, d->total_ctrl);
    arr(d->points, (size_t)d->total_points * 8);
    arr(d->thickness, (size_t)d->total_points * 4);
    arr(d->group_shape_offset, ng * 4);
    arr(d->group_shape_count, ng * 4);
    arr(d->group_shape_ids, (size_t)d->total_group_shapes * 4);
    arr(d->group_fill_rule, ng * 4);
    arr(d->group_shape_to_canvas, ng * 36);
    arr(d->group_canvas_to_shape, ng * 36);
    arr(d->group_fill_paint, ng * 4);
    arr(d->group_stroke_paint, ng * 4);
    arr(d->paint_kind, np * 4);
    arr(d->paint_params, np * 16);
    arr(d->paint_stop_offset, np * 4);
    arr(d->paint_stop_count, np * 4);
    arr(d->stop_offsets, (size_t)d->total_stops * 4);
    arr(d->stop_colors, (size_t)d->total_stops * 16);
}

dvg_status check_options(const dvg_render_options* o) {
    if (!o) return fail(DVG_ERR_INVALID_ARGUMENT, "null render options");
    return DVG_OK;
}
SampleParams sample_params(const dvg_render_options* o, const dvg_tuning& tune) {
    SampleParams sp;
    sp.layout = (int)tune.sample_layout;
    sp.fwd_occ = (int)tune.forward_occupancy;
    sp.sxn = o->samples_x > 0 ? (int)o->samples_x : 1;
    sp.syn = o->samples_y > 0 ? (int)o->samples_y : 1;
    sp.seed = o->seed;
    sp.jitter = o->jitter != 0 && o->use_prefiltering == 0;
    sp.frag = nullptr;
    sp.frag_n = nullptr;
    sp.frag_slots = 0;
    sp.tile_base = 0;
    sp.tile_count = 0;
    return sp;
}
// Points sp at a fragment cache of frag_cache_bytes(tiles, spp, slots) bytes at `base`.
void attach_frag(SampleParams& sp, void* base, int tiles, int slots) {
    const size_t samples = (size_t)tiles * sp.sxn * sp.syn * 256;
    sp.frag = static_cast<uint16_t*>(base);
    sp.frag_n = reinterpret_cast<uint8_t*>(sp.frag + samples * (size_t)slots);
    sp.frag_slots = slots;
}
dvg_status check_status(dvg_context* ctx) {
    unsigned st = 0;
    CK(cudaMemcpyAsync(&st, ctx->status, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (st & ST_FRAGMENT_OVERFLOW) {
        CK(cudaMemsetAsync(ctx->status, 0, sizeof(unsigned), ctx->stream));
        return fail(DVG_ERR_DEVICE_LIMIT, "a sample covered more fragments than the per-thread capacity (" +
                                              std::to_string(MAX_FRAGMENTS) + ")");
    }
    if (st & ST_BVH_LIMIT) {
        CK(cudaMemsetAsync(ctx->status, 0, sizeof(unsigned), ctx->stream));
        return fail(DVG_ERR_DEVICE_LIMIT, "a BVH traversal exceeded its stack depth");
    }
    if (st & ST_REFIT_LAYOUT) {
        CK(cudaMemsetAsync(ctx->status, 0, sizeof(unsigned), ctx->stream));
        return fail(DVG_ERR_LAUNCH, "on-device scene re-preparation found a BVH layout it did not build");
    }
    return DVG_OK;
}

// Brackets one launcher call with CUDA events on the context stream when profiling is on.
struct Prof {
    dvg_context* ctx;
    ProfEvent ev{};
    Prof(dvg_context* c, const char* name) : ctx(c) {
        ev.name = name;
        if (!ctx->profiling) return;
        cudaEventCreate(&ev.a);
        cudaEventCreate(&ev.b);
        cudaEventRecord(ev.a, ctx->stream);
    }
    ~Prof() {
        if (!ctx->profiling) return;
        cudaEventRecord(ev.b, ctx->stream);
        ctx->pending.push_back(ev);
    }
};
void resolve_profile(dvg_context* ctx) {
    for (auto& e : ctx->pending) {
        cudaEventSynchronize(e.b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e.a, e.b);
        bool found = false;
        for (auto& st : ctx->stats)
            if (std::strcmp(st.name, e.name) == 0) {
                st.ms += ms;
                st.count += 1;
                found = true;
            }
        if (!found) ctx->stats.push_back(ProfStat{e.name, (double)ms, 1});
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    ctx->pending.clear();
}

}  // namespace

extern "C" {

dvg_status dvg_context_set_profiling(dvg_context* ctx, int enable) {
    if (!ctx) return fail(DVG_ERR_INVALID_ARGUMENT, "null context");
    ctx->profiling = enable != 0;
    return DVG_OK;
}

int dvg_context_profile(dvg_context* ctx, const char** names, double* total_ms, uint64_t* launches, int cap) {
    if (!ctx) return 0;
    cudaSetDevice(ctx->device);
    resolve_profile(ctx);
    int n = (int)ctx->stats.size();
    for (int i = 0; i < n && i < cap; ++i) {
        if (names) names[i] = ctx->stats[i].name;
        if (total_ms) total_ms[i] = ctx->stats[i].ms;
        if (launches) launches[i] = ctx->stats[i].count;
    }
    return n;
}

void dvg_context_profile_reset(dvg_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    resolve_profile(ctx);
    ctx->stats.clear();
}


uint32_t dvg_abi_version(void) { return DVG_ABI_VERSION; }

const char* dvg_last_error(void) { return g_last_error.c_str(); }

dvg_status dvg_context_create(int device, dvg_context** out) {
    if (!out) return fail(DVG_ERR_INVALID_ARGUMENT, "null output pointer");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(DVG_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= count) return fail(DVG_ERR_INVALID_ARGUMENT, "device index out of range");
    std::unique_ptr<dvg_context> ctx(new dvg_context());
    ctx->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaMalloc(&ctx->status, sizeof(unsigned)));
    CK(cudaMemsetAsync(ctx->status, 0, sizeof(unsigned), ctx->stream));
    *out = ctx.release();
    return DVG_OK;
}

dvg_status dvg_context_set_retain(dvg_context* ctx, int enable) {
    if (!ctx) return fail(DVG_ERR_INVALID_ARGUMENT, "null context");
    ctx->retain = enable != 0;
    if (!ctx->retain && ctx->kept) {
        CK(cudaSetDevice(ctx->device));
        dvg_scene_destroy(ctx->kept);
        ctx->kept = nullptr;
    }
    return DVG_OK;
}

void dvg_context_destroy(dvg_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->kept) dvg_scene_destroy(ctx->kept);
    ctx->kept = nullptr;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->status) cudaFree(ctx->status);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

uint64_t dvg_context_launch_count(const dvg_context* ctx) { return ctx ? ctx->launches : 0; }

void* dvg_context_stream(dvg_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

dvg_status dvg_scene_upload(dvg_context* ctx, const dvg_scene_desc* desc, dvg_scene** out) {
    if (!ctx || !desc || !out) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    std::unique_ptr<dvg_scene> sc(new dvg_scene());
    sc->ctx = ctx;
    std::string err;
    dvg_status st = prepare_scene(desc, &sc->host, &err);
    if (st != DVG_OK) return fail(st, err);
    const HostScene& h = sc->host;
    Blob b;
    size_t o_g_c2s = b.add(h.g_c2s), o_g_s2c = b.add(h.g_s2c), o_g_info = b.add(h.g_info), o_g_bvh = b.add(h.g_bvh),
           o_g_bbox = b.add(h.g_bbox), o_g_list = b.add(h.g_shape_list), o_gn_b = b.add(h.gn_bounds),
           o_gn_m = b.add(h.gn_meta), o_gl = b.add(h.gl_shapes), o_s_info = b.add(h.s_info),
           o_s_prm = b.add(h.s_params), o_s_inv = b.add(h.s_inv), o_s_x = b.add(h.s_xform),
           o_s_sw = b.add(h.s_stroke), o_s_box = b.add(h.s_box), o_s_pm = b.add(h.s_padmul),
           o_p_shape = b.add(h.p_shape), o_p_miter = b.add(h.p_miter), o_p_info = b.add(h.p_info),
           o_pn_b = b.add(h.pn_bounds),
           o_pn_m = b.add(h.pn_meta), o_pl = b.add(h.pl_segs), o_seg_p = b.add(h.seg_p), o_seg_r = b.add(h.seg_r),
           o_seg_m = b.add(h.seg_meta), o_pts = b.add(h.points), o_th = b.add(h.thickness), o_ncp = b.add(h.ncp),
           o_pi = b.add(h.paint_info), o_pp = b.add(h.paint_params), o_so = b.add(h.stop_offsets),
           o_sc = b.add(h.stop_colors), o_len = b.add(h.shape_len), o_bcdf = b.add(h.bcdf),
           o_bpmf = b.add(h.bpmf), o_bs = b.add(h.b_shape), o_bg = b.add(h.b_group),
           o_pci = b.add(h.path_cdf_info), o_pcdf = b.add(h.path_cdf), o_ppmf = b.add(h.path_pmf),
           o_ppid = b.add(h.path_pid), o_plen = b.add(h.path_len_arr), o_bgi = b.add(h.bg_image);
    CK(sc->arena.reserve(b.data.size()));
    sc->arena_bytes = b.data.size();
    CK(cudaMemcpyAsync(sc->arena.ptr, b.data.data(), b.data.size(), cudaMemcpyHostToDevice, ctx->stream));
    char* base = sc->arena.as<char>();
    DevScene& S = sc->dev;
    S.width = (int)h.width;
    S.height = (int)h.height;
    S.num_groups = (int)h.num_groups;
    S.num_shapes = (int)h.num_shapes;
    S.num_paints = (int)h.num_paints;
    S.num_paths = (int)h.num_paths;
    S.filter_type = (int)h.filter_type;
    S.filter_radius = h.filter_radius;
    {
        float c = std::ceil(h.filter_radius);
        S.filter_ri = c > 0.0f ? (int)std::min(c, 1024.0f) : 0;
    }
    for (int k = 0; k < 4; ++k) S.bg[k] = h.bg[k];
    S.bg_image = h.bg_image.empty() ? nullptr : (const float*)(base + o_bgi);
    S.g_c2s = (const float*)(base + o_g_c2s);
    S.g_s2c = (const float*)(base + o_g_s2c);
    S.g_info = (const int4*)(base + o_g_info);
    S.g_bvh = (const int4*)(base + o_g_bvh);
    S.g_shape_list = (const int*)(base + o_g_list);
    S.gn_bounds = (const float4*)(base + o_gn_b);
    S.gn_meta = (const int4*)(base + o_gn_m);
    S.gl_shapes = (const int*)(base + o_gl);
    S.s_info = (const int4*)(base + o_s_info);
    S.s_params = (const float4*)(base + o_s_prm);
    S.s_inv = (const float*)(base + o_s_inv);
    S.s_xform = (const float*)(base + o_s_x);
    S.s_stroke = (const float*)(base + o_s_sw);
    S.s_box = (const float4*)(base + o_s_box);
    S.s_padmul = (const float*)(base + o_s_pm);
    S.p_shape = (const int*)(base + o_p_shape);
    S.p_miter = (const float*)(base + o_p_miter);
    S.styled = h.any_styled ? 1 : 0;
    S.p_info = (const int4*)(base + o_p_info);
    S.pn_bounds = (const float4*)(base + o_pn_b);
    S.pn_meta = (const int4*)(base + o_pn_m);
    S.pl_segs = (const int*)(base + o_pl);
    S.seg_p = (const float4*)(base + o_seg_p);
    S.seg_r = (const float4*)(base + o_seg_r);
    S.seg_meta = (const int4*)(base + o_seg_m);
    S.points = (const float2*)(base + o_pts);
    S.thickness = (const float*)(base + o_th);
    S.ncp = (const uint8_t*)(base + o_ncp);
    S.paint_info = (const int4*)(base + o_pi);
    S.paint_params = (const float4*)(base + o_pp);
    S.stop_offsets = (const float*)(base + o_so);
    S.stop_colors = (const float4*)(base + o_sc);
    S.boundary_ok = h.boundary_ok ? 1 : 0;
    S.bcdf_n = (int)h.bcdf.size();
    S.shape_len = (const float*)(base + o_len);
    S.bcdf = (const float*)(base + o_bcdf);
    S.bpmf = (const float*)(base + o_bpmf);
    S.b_shape = (const int*)(base + o_bs);
    S.b_group = (const int*)(base + o_bg);
    S.path_cdf_info = (const int4*)(base + o_pci);
    S.path_cdf = (const float*)(base + o_pcdf);
    S.path_pmf = (const float*)(base + o_ppmf);
    S.path_pid = (const int*)(base + o_ppid);
    S.path_len = (const float*)(base + o_plen);
    sc->g_bbox = (const float4*)(base + o_g_bbox);
    S.g_bbox = sc->g_bbox;
    // tile binning
    S.tiles_x = (S.width + TILE - 1) / TILE;
    S.tiles_y = (S.height + TILE - 1) / TILE;
    const int tiles = S.tiles_x * S.tiles_y;
    if (tiles > 0) {
        CK(sc->tiles.reserve(sizeof(int) * (2 * (size_t)tiles + 1)));
        int* counts = sc->tiles.as<int>();
        int* offsets = counts + tiles;
        ctx->launches += launch_binning(S, sc->g_bbox, counts, offsets, nullptr, ctx->stream);
        CK(cudaGetLastError());
        int total = 0;
        CK(cudaMemcpyAsync(&total, offsets + tiles, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        CK(sc->entries.reserve(sizeof(int) * (size_t)std::max(total, 1)));
        S.tile_offsets = offsets;
        S.tile_entries = sc->entries.as<int>();
        ctx->launches += launch_binning(S, sc->g_bbox, counts, offsets, sc->entries.as<int>(), ctx->stream);
        CK(cudaGetLastError());
    }
    layout_grads(sc.get());
    CK(sc->grads.reserve(sizeof(float) * std::max<size_t>(sc->grad_floats, 64)));
    CK(cudaStreamSynchronize(ctx->stream));
    *out = sc.release();
    return DVG_OK;
}

void dvg_scene_destroy(dvg_scene* scene) {
    if (!scene) return;
    cudaSetDevice(scene->ctx->device);
    cudaStreamSynchronize(scene->ctx->stream);
    if (scene->ctx->shard_scene == scene) scene->ctx->shard_scene = nullptr;
    delete scene;
}

// `frag_out` non-null: the forward also fills the context's fragment cache for the
// interior pass that follows (non-prefiltered, cache enabled by the scene's tuning);
// *frag_out tells whether it did.
// *weights_out: whether ctx->wsum now holds this scene's weight image.
static dvg_status render_into(dvg_context* ctx, dvg_scene* sc, const dvg_render_options* opts, float* out_dev,
                              bool* frag_out = nullptr, bool* weights_out = nullptr) {
    const DevScene& S = sc->dev;
    if (frag_out) *frag_out = false;
    if (weights_out) *weights_out = false;
    const size_t npix = (size_t)S.width * S.height;
    if (npix == 0) return DVG_OK;
    if (S.num_groups == 0) {  // Image::solid / background image (src/renderer/renderer.rs:57-66)
        {
            Prof prof_(ctx, "fill_background");
            ctx->launches += launch_fill_background(S, out_dev, ctx->stream);
        }
        CK(cudaGetLastError());
        return DVG_OK;
    }
    ++ctx->gen;  // accum, wsum and the fragment cache are rewritten below
    SampleParams sp = sample_params(opts, sc->tune);
    if (frag_out && !opts->use_prefiltering && sc->tune.fragment_slots > 0) {
        const int tiles = S.tiles_x * S.tiles_y, slots = (int)sc->tune.fragment_slots;
        CK(ctx->frag.reserve(frag_cache_bytes(tiles, sp.sxn * sp.syn, slots)));
        attach_frag(sp, ctx->frag.ptr, tiles, slots);
        *frag_out = true;
    }
    CK(ctx->accum.reserve(npix * 4 * sizeof(float)));
    CK(ctx->wsum.reserve(npix * sizeof(float)));
    CK(cudaMemsetAsync(ctx->accum.ptr, 0, npix * 4 * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(ctx->wsum.ptr, 0, npix * sizeof(float), ctx->stream));
    {
        Prof prof_(ctx, opts->use_prefiltering ? "forward_prefilter" : "forward");
        if (opts->use_prefiltering)
            ctx->launches += launch_forward_prefilter(S, sp, ctx->accum.as<float>(), ctx->wsum.as<float>(), ctx->status,
                                                      ctx->stream);
        else
            ctx->launches += launch_forward(S, sp, ctx->accum.as<float>(), ctx->wsum.as<float>(), ctx->status,
                                            ctx->stream);
    }
    CK(cudaGetLastError());
    {
        Prof prof_(ctx, "resolve");
        ctx->launches += launch_resolve(S, ctx->accum.as<float>(), ctx->wsum.as<float>(), out_dev, ctx->stream);
    }
    CK(cudaGetLastError());
    if (weights_out) *weights_out = true;
    return DVG_OK;
}

dvg_status dvg_render_device(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts, float* out_rgba) {
    if (!ctx || !scene || !out_rgba) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    return render_into(ctx, scene, opts, out_rgba);
}

static dvg_status render_host_impl(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                   float* out_rgba, bool* frag_out, bool* weights_out);
dvg_status dvg_render_host(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts, float* out_rgba) {
    return render_host_impl(ctx, scene, opts, out_rgba, nullptr, nullptr);
}
static dvg_status render_host_impl(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                   float* out_rgba, bool* frag_out, bool* weights_out) {
    if (frag_out) *frag_out = false;
    if (weights_out) *weights_out = false;
    if (!ctx || !scene || !out_rgba) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    const HostScene& h = scene->host;
    const size_t npix = (size_t)h.width * h.height;
    if (npix == 0) return DVG_OK;
    if (h.num_groups == 0) {  // src/renderer/renderer.rs:57-66
        for (size_t i = 0; i < npix; ++i)
            for (int k = 0; k < 4; ++k) out_rgba[4 * i + k] = h.bg_image.empty() ? h.bg[k] : h.bg_image[4 * i + k];
        return DVG_OK;
    }
    CK(ctx->image.reserve(npix * 4 * sizeof(float)));
    st = render_into(ctx, scene, opts, ctx->image.as<float>(), frag_out, weights_out);
    if (st != DVG_OK) return st;
    CK(cudaMemcpyAsync(out_rgba, ctx->image.ptr, npix * 4 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

// Backward on device buffers.  `have_weights`: ctx->wsum already holds this scene's
// weights; `frag_ready`: the forward just filled ctx->frag for these options.
// `shard` (optional): only its tiles and boundary samples, with the weight image
// `shard_wsum` (the sum over all shards' forwards) instead of ctx->wsum.
static dvg_status backward_core(dvg_context* ctx, dvg_scene* sc, const dvg_render_options* opts,
                                const dvg_backward_options* bopts, const float* d_render, const float* d_sdf,
                                const GradPtrs& G, bool have_weights, bool frag_ready = false,
                                const dvg_shard* shard = nullptr, const float* shard_wsum = nullptr) {
    const DevScene& S = sc->dev;
    const size_t npix = (size_t)S.width * S.height;
    if (npix == 0) return DVG_OK;
    SampleParams sp = sample_params(opts, sc->tune);
    if (frag_ready) attach_frag(sp, ctx->frag.ptr, S.tiles_x * S.tiles_y, (int)sc->tune.fragment_slots);
    const bool run_tiles = !shard || shard->tile_end > shard->tile_begin;  // a shard may hold samples only
    if (shard && run_tiles) {
        sp.tile_base = (int)shard->tile_begin;
        sp.tile_count = (int)(shard->tile_end - shard->tile_begin);
    }
    // read at each launch: the weights pass below may (re)allocate ctx->wsum
    auto wsum_now = [&]() -> const float* { return shard ? shard_wsum : ctx->wsum.as<float>(); };
    if (d_render && S.num_groups > 0) {
        if (!have_weights) {
            ++ctx->gen;
            CK(ctx->wsum.reserve(npix * sizeof(float)));
            CK(cudaMemsetAsync(ctx->wsum.ptr, 0, npix * sizeof(float), ctx->stream));
            Prof prof_(ctx, "weights");
            ctx->launches += launch_weights(S, sp, ctx->wsum.as<float>(), ctx->stream);
            CK(cudaGetLastError());
        }
        if (run_tiles) {
            Prof prof_(ctx, opts->use_prefiltering ? "interior_prefilter" : "interior");
            if (opts->use_prefiltering)
                ctx->launches +=
                    launch_interior_prefilter(S, sp, d_render, wsum_now(), G, ctx->status, ctx->stream);
            else
                ctx->launches += launch_interior(S, sp, d_render, wsum_now(), G, ctx->status, ctx->stream);
        }
        CK(cudaGetLastError());
        if (S.boundary_ok && !opts->use_prefiltering) {  // src/backward/render.rs:191
            BoundaryParams bp;
            uint64_t total = (uint64_t)npix * sp.sxn * sp.syn;
            total = bopts && bopts->boundary_samples ? bopts->boundary_samples : total;
            bp.sample_base = shard ? std::min<uint64_t>(shard->sample_begin, total) : 0;
            bp.num_samples = shard ? std::min<uint64_t>(std::max(shard->sample_end, shard->sample_begin), total) : total;
            bp.slot_base = bp.sample_base;
            bp.pdf_scale = (float)((double)total / (double)((uint64_t)npix * sp.sxn * sp.syn));
            bp.seed = (bopts && !bopts->boundary_seed_from_options) ? bopts->boundary_seed : opts->seed;
            bp.rng = bopts ? (int)bopts->rng : 0;
            bp.cell = (int)sc->tune.boundary_cell;
            const uint64_t cap = std::max<uint64_t>(std::min<uint64_t>(bp.num_samples - bp.sample_base, (uint64_t)1 << 24), 1);
            const int tiles = S.tiles_x * S.tiles_y;
            CK(ctx->bsamples.reserve(cap * sizeof(BSample)));
            CK(ctx->bkey.reserve(cap * sizeof(int)));
            CK(ctx->border.reserve(cap * sizeof(int)));
            CK(ctx->bcounts.reserve(bnd_count_ints((size_t)tiles) * sizeof(int)));
            Prof prof_(ctx, "boundary");
            ctx->launches += launch_boundary(S, bp, d_render, wsum_now(), G, ctx->bsamples.as<BSample>(),
                                             ctx->bkey.as<int>(), ctx->bcounts.as<int>(), ctx->border.as<int>(), cap,
                                             ctx->stream);
            CK(cudaGetLastError());
        }
    } else if (d_render && S.num_groups == 0) {
        // only the background receives gradient: every sample lands on it.
        if (!have_weights) {
            ++ctx->gen;
            CK(ctx->wsum.reserve(npix * sizeof(float)));
            CK(cudaMemsetAsync(ctx->wsum.ptr, 0, npix * sizeof(float), ctx->stream));
            Prof prof_(ctx, "weights");
            ctx->launches += launch_weights(S, sp, ctx->wsum.as<float>(), ctx->stream);
        }
        if (run_tiles) {
            Prof prof_(ctx, "interior");
            ctx->launches += launch_interior(S, sp, d_render, wsum_now(), G, ctx->status, ctx->stream);
        }
        CK(cudaGetLastError());
    }
    if (d_sdf && S.num_groups > 0) {  // the d_sdf_image part (src/renderer/backward_gpu.rs:512-520)
        Prof prof_(ctx, "sdf_backward");
        ctx->launches += launch_sdf_backward(S, sp, d_sdf, G, bopts && bopts->compute_translation && G.d_translation,
                                             ctx->status, ctx->stream);
        CK(cudaGetLastError());
    }
    {
        Prof prof_(ctx, "finalize_background");
        ctx->launches += launch_finalize_background(S, G, ctx->stream);
    }
    CK(cudaGetLastError());
    return DVG_OK;
}

static GradPtrs grads_from_user(const dvg_grads* g) {
    GradPtrs p;
    p.d_shape_params = g->d_shape_params;
    p.d_shape_transform = g->d_shape_transform;
    p.d_shape_stroke_width = g->d_shape_stroke_width;
    p.d_points = g->d_points;
    p.d_thickness = g->d_thickness;
    p.d_group_transform = g->d_group_transform;
    p.d_paint_params = g->d_paint_params;
    p.d_stop_offsets = g->d_stop_offsets;
    p.d_stop_colors = g->d_stop_colors;
    p.d_filter_radius = g->d_filter_radius;
    p.d_background = g->d_background;
    p.d_background_image = g->d_background_image;
    p.d_translation = g->d_translation;
    return p;
}

// Zero every part of a device gradient set (scene arena or caller buffers).
static dvg_status zero_grads(dvg_context* ctx, dvg_scene* sc, const GradPtrs& G) {
    const HostScene& h = sc->host;
    const size_t npix = (size_t)h.width * h.height;
    struct Part {
        float* p;
        size_t n;
    } parts[] = {{G.d_shape_params, 4 * (size_t)h.num_shapes},
                 {G.d_shape_transform, 9 * (size_t)h.num_shapes},
                 {G.d_shape_stroke_width, h.num_shapes},
                 {G.d_points, 2 * (size_t)h.total_points},
                 {G.d_thickness, h.total_points},
                 {G.d_group_transform, 9 * (size_t)h.num_groups},
                 {G.d_paint_params, 4 * (size_t)h.num_paints},
                 {G.d_stop_offsets, h.total_stops},
                 {G.d_stop_colors, 4 * (size_t)h.total_stops},
                 {G.d_filter_radius, 1},
                 {G.d_background, 4},
                 {G.d_background_image, 4 * npix},
                 {G.d_translation, 2 * npix}};
    for (auto& p : parts)
        if (p.p && p.n) CK(cudaMemsetAsync(p.p, 0, p.n * sizeof(float), ctx->stream));
    return DVG_OK;
}

static dvg_status check_backward_args(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                      const float* d_sdf, const dvg_grads* grads) {
    if (!ctx || !scene || !grads) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    const GradPtrs G = grads_from_user(grads);
    if (!G.d_shape_params || !G.d_shape_transform || !G.d_shape_stroke_width || !G.d_group_transform ||
        !G.d_paint_params || !G.d_filter_radius || !G.d_background ||
        (scene->host.total_points && (!G.d_points || !G.d_thickness)) ||
        (scene->host.total_stops && (!G.d_stop_offsets || !G.d_stop_colors)))
        return fail(DVG_ERR_INVALID_ARGUMENT, "missing gradient buffer");
    return DVG_OK;
}

dvg_status dvg_render_backward_device(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                      const dvg_backward_options* bopts, const float* d_render, const float* d_sdf,
                                      dvg_grads* grads) {
    dvg_status st = check_backward_args(ctx, scene, opts, d_sdf, grads);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    GradPtrs G = grads_from_user(grads);
    if (!(bopts && bopts->compute_translation)) G.d_translation = nullptr;
    if (!(d_render && scene->dev.bg_image)) G.d_background_image = nullptr;
    st = zero_grads(ctx, scene, grads_from_user(grads));
    if (st != DVG_OK) return st;
    return backward_core(ctx, scene, opts, bopts, d_render, d_sdf, G, false);
}

static dvg_status backward_host_impl(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                     const dvg_backward_options* bopts, const float* d_render, const float* d_sdf,
                                     dvg_grads* grads, bool have_weights, bool frag_ready);
dvg_status dvg_render_backward_host(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                    const dvg_backward_options* bopts, const float* d_render, const float* d_sdf,
                                    dvg_grads* grads) {
    return backward_host_impl(ctx, scene, opts, bopts, d_render, d_sdf, grads, false, false);
}
static dvg_status backward_host_impl(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                     const dvg_backward_options* bopts, const float* d_render, const float* d_sdf,
                                     dvg_grads* grads, bool have_weights, bool frag_ready) {
    dvg_status st = check_backward_args(ctx, scene, opts, d_sdf, grads);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    const HostScene& h = scene->host;
    const size_t npix = (size_t)h.width * h.height;
    GradPtrs G = device_grads(scene);
    CK(cudaMemsetAsync(scene->grads.ptr, 0, scene->grad_floats * sizeof(float), ctx->stream));
    bool want_bg_img = d_render && !h.bg_image.empty() && grads->d_background_image;
    bool want_tr = bopts && bopts->compute_translation && grads->d_translation;
    if (want_bg_img) {
        CK(ctx->bg_grad.reserve(npix * 4 * sizeof(float)));
        CK(cudaMemsetAsync(ctx->bg_grad.ptr, 0, npix * 4 * sizeof(float), ctx->stream));
        G.d_background_image = ctx->bg_grad.as<float>();
    }
    if (want_tr) {
        CK(ctx->trans_grad.reserve(npix * 2 * sizeof(float)));
        CK(cudaMemsetAsync(ctx->trans_grad.ptr, 0, npix * 2 * sizeof(float), ctx->stream));
        G.d_translation = ctx->trans_grad.as<float>();
    }
    const float* dr = nullptr;
    if (d_render && npix) {
        CK(ctx->d_render.reserve(npix * 4 * sizeof(float)));
        CK(cudaMemcpyAsync(ctx->d_render.ptr, d_render, npix * 4 * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
        dr = ctx->d_render.as<float>();
    }
    const float* ds = nullptr;
    if (d_sdf && npix) {
        CK(ctx->sdf.reserve(npix * sizeof(float)));
        CK(cudaMemcpyAsync(ctx->sdf.ptr, d_sdf, npix * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        ds = ctx->sdf.as<float>();
    }
    st = backward_core(ctx, scene, opts, bopts, dr, ds, G, have_weights, frag_ready);
    if (st != DVG_OK) return st;
    struct Part {
        float* dst;
        const float* src;
        size_t n;
    } parts[] = {{grads->d_shape_params, G.d_shape_params, 4 * (size_t)h.num_shapes},
                 {grads->d_shape_transform, G.d_shape_transform, 9 * (size_t)h.num_shapes},
                 {grads->d_shape_stroke_width, G.d_shape_stroke_width, h.num_shapes},
                 {grads->d_points, G.d_points, 2 * (size_t)h.total_points},
                 {grads->d_thickness, G.d_thickness, h.total_points},
                 {grads->d_group_transform, G.d_group_transform, 9 * (size_t)h.num_groups},
                 {grads->d_paint_params, G.d_paint_params, 4 * (size_t)h.num_paints},
                 {grads->d_stop_offsets, G.d_stop_offsets, h.total_stops},
                 {grads->d_stop_colors, G.d_stop_colors, 4 * (size_t)h.total_stops},
                 {grads->d_filter_radius, G.d_filter_radius, 1},
                 {grads->d_background, G.d_background, 4}};
    for (auto& p : parts)
        if (p.dst && p.n) CK(cudaMemcpyAsync(p.dst, p.src, p.n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (grads->d_background_image) {
        if (want_bg_img)
            CK(cudaMemcpyAsync(grads->d_background_image, G.d_background_image, npix * 4 * sizeof(float),
                               cudaMemcpyDeviceToHost, ctx->stream));
        else
            std::memset(grads->d_background_image, 0, npix * 4 * sizeof(float));
    }
    if (grads->d_translation) {
        if (want_tr)
            CK(cudaMemcpyAsync(grads->d_translation, G.d_translation, npix * 2 * sizeof(float),
                               cudaMemcpyDeviceToHost, ctx->stream));
        else
            std::memset(grads->d_translation, 0, npix * 2 * sizeof(float));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

dvg_status dvg_render(dvg_context* ctx, const dvg_scene_desc* desc, const dvg_render_options* opts, float* out_rgba) {
    if (!ctx || !desc || !out_rgba) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    dvg_scene* sc = nullptr;
    st = dvg_scene_upload(ctx, desc, &sc);
    if (st != DVG_OK) return st;
    if (!ctx->retain) {
        st = dvg_render_host(ctx, sc, opts, out_rgba);
        dvg_scene_destroy(sc);
        return st;
    }
    bool frag = false, weights = false;
    st = render_host_impl(ctx, sc, opts, out_rgba, &frag, &weights);
    if (ctx->kept) dvg_scene_destroy(ctx->kept);
    ctx->kept = nullptr;
    if (st != DVG_OK) {
        dvg_scene_destroy(sc);
        return st;
    }
    ctx->kept = sc;
    desc_key(desc, ctx->kept_key);
    ctx->kept_opts = *opts;
    ctx->kept_gen = ctx->gen;
    ctx->kept_weights = weights;
    ctx->kept_frag = frag;
    return st;
}

dvg_status dvg_render_backward(dvg_context* ctx, const dvg_scene_desc* desc, const dvg_render_options* opts,
                               const dvg_backward_options* bopts, const float* d_render, const float* d_sdf,
                               dvg_grads* grads) {
    if (!ctx || !desc || !grads) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    if (ctx->retain && ctx->kept && ctx->kept_gen == ctx->gen &&
        std::memcmp(&ctx->kept_opts, opts, sizeof(dvg_render_options)) == 0) {
        std::vector<char> key;
        desc_key(desc, key);
        if (key == ctx->kept_key)  // the scene, weights and fragments of the last dvg_render
            return backward_host_impl(ctx, ctx->kept, opts, bopts, d_render, d_sdf, grads, ctx->kept_weights,
                                      ctx->kept_frag);
    }
    dvg_scene* sc = nullptr;
    st = dvg_scene_upload(ctx, desc, &sc);
    if (st != DVG_OK) return st;
    st = dvg_render_backward_host(ctx, sc, opts, bopts, d_render, d_sdf, grads);
    dvg_scene_destroy(sc);
    return st;
}

dvg_status dvg_fwd_bwd_l2_device(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                 const dvg_backward_options* bopts, const float* target_rgba, float* out_rgba,
                                 float* loss_out, dvg_grads* grads) {
    dvg_status st = check_backward_args(ctx, scene, opts, nullptr, grads);
    if (st != DVG_OK) return st;
    if (!target_rgba) return fail(DVG_ERR_INVALID_ARGUMENT, "null target");
    CK(cudaSetDevice(ctx->device));
    const size_t npix = (size_t)scene->dev.width * scene->dev.height;
    if (npix == 0) return DVG_OK;
    float* img = out_rgba;
    if (!img) {
        CK(ctx->image.reserve(npix * 4 * sizeof(float)));
        img = ctx->image.as<float>();
    }
    bool frag = false;
    st = render_into(ctx, scene, opts, img, &frag);
    if (st != DVG_OK) return st;
    CK(ctx->d_render.reserve(npix * 4 * sizeof(float)));
    if (loss_out) CK(cudaMemsetAsync(loss_out, 0, sizeof(float), ctx->stream));
    {
        Prof prof_(ctx, "l2_loss");
        ctx->launches += launch_l2(img, target_rgba, npix * 4, ctx->d_render.as<float>(), loss_out, ctx->stream);
    }
    CK(cudaGetLastError());
    GradPtrs G = grads_from_user(grads);
    if (!(bopts && bopts->compute_translation)) G.d_translation = nullptr;
    if (!scene->dev.bg_image) G.d_background_image = nullptr;
    st = zero_grads(ctx, scene, G);
    if (st != DVG_OK) return st;
    return backward_core(ctx, scene, opts, bopts, ctx->d_render.as<float>(), nullptr, G, true, frag);
}

// ---------------------------------------------------------------------------
// One scene split over several processes: forward per band of tiles, the caller sums
// the accumulators, then resolve / loss on the whole image and backward per band of
// tiles and range of boundary samples; the caller sums the gradients.
static dvg_status check_shard(const dvg_scene* scene, const dvg_shard* shard) {
    if (!shard) return fail(DVG_ERR_INVALID_ARGUMENT, "null shard");
    const uint32_t tiles = (uint32_t)(scene->dev.tiles_x * scene->dev.tiles_y);
    if (shard->tile_begin > shard->tile_end || shard->tile_end > tiles || shard->sample_begin > shard->sample_end)
        return fail(DVG_ERR_INVALID_ARGUMENT, "shard range out of order or past the last tile");
    return DVG_OK;
}

dvg_status dvg_scene_tile_count(const dvg_scene* scene, uint32_t* tiles) {
    if (!scene || !tiles) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    *tiles = (uint32_t)(scene->dev.tiles_x * scene->dev.tiles_y);
    return DVG_OK;
}

dvg_status dvg_scene_tile_groups(const dvg_scene* scene, uint32_t* groups, uint32_t n) {
    if (!scene || !groups) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    const uint32_t tiles = (uint32_t)(scene->dev.tiles_x * scene->dev.tiles_y);
    if (n < tiles) return fail(DVG_ERR_INVALID_ARGUMENT, "buffer holds fewer entries than the scene has tiles");
    if (tiles == 0) return DVG_OK;
    CK(cudaSetDevice(scene->ctx->device));
    std::vector<int> off(tiles + 1, 0);
    CK(cudaMemcpyAsync(off.data(), scene->dev.tile_offsets, (tiles + 1) * sizeof(int), cudaMemcpyDeviceToHost,
                       scene->ctx->stream));
    CK(cudaStreamSynchronize(scene->ctx->stream));
    for (uint32_t t = 0; t < tiles; ++t) groups[t] = (uint32_t)(off[t + 1] - off[t]);
    return DVG_OK;
}

dvg_status dvg_shard_forward(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                             const dvg_shard* shard, float* accum_rgba, float* wsum) {
    if (!ctx || !scene || !accum_rgba || !wsum) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st == DVG_OK) st = check_shard(scene, shard);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    const DevScene& S = scene->dev;
    const size_t npix = (size_t)S.width * S.height;
    ++ctx->gen;
    ctx->shard_scene = nullptr;
    if (npix == 0) return DVG_OK;
    CK(cudaMemsetAsync(accum_rgba, 0, npix * 4 * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(wsum, 0, npix * sizeof(float), ctx->stream));
    if (S.num_groups == 0 || shard->tile_end == shard->tile_begin) return DVG_OK;
    SampleParams sp = sample_params(opts, scene->tune);
    sp.tile_base = (int)shard->tile_begin;
    sp.tile_count = (int)(shard->tile_end - shard->tile_begin);
    bool frag = false;
    if (!opts->use_prefiltering && scene->tune.fragment_slots > 0) {
        const int tiles = S.tiles_x * S.tiles_y, slots = (int)scene->tune.fragment_slots;
        CK(ctx->frag.reserve(frag_cache_bytes(tiles, sp.sxn * sp.syn, slots)));
        attach_frag(sp, ctx->frag.ptr, tiles, slots);
        frag = true;
    }
    {
        Prof prof_(ctx, opts->use_prefiltering ? "forward_prefilter" : "forward");
        if (opts->use_prefiltering)
            ctx->launches += launch_forward_prefilter(S, sp, accum_rgba, wsum, ctx->status, ctx->stream);
        else
            ctx->launches += launch_forward(S, sp, accum_rgba, wsum, ctx->status, ctx->stream);
    }
    CK(cudaGetLastError());
    ctx->shard_scene = scene;
    ctx->shard_opts = *opts;
    ctx->shard_t0 = shard->tile_begin;
    ctx->shard_t1 = shard->tile_end;
    ctx->shard_gen = ctx->gen;
    ctx->shard_frag = frag;
    ctx->shard_tune = scene->tune;
    return DVG_OK;
}

dvg_status dvg_shard_resolve(dvg_context* ctx, dvg_scene* scene, const float* accum_rgba, const float* wsum,
                             float* out_rgba) {
    if (!ctx || !scene || !accum_rgba || !wsum || !out_rgba) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    const DevScene& S = scene->dev;
    if ((size_t)S.width * S.height == 0) return DVG_OK;
    if (S.num_groups == 0) {
        ctx->launches += launch_fill_background(S, out_rgba, ctx->stream);
    } else {
        Prof prof_(ctx, "resolve");
        ctx->launches += launch_resolve(S, accum_rgba, wsum, out_rgba, ctx->stream);
    }
    CK(cudaGetLastError());
    return DVG_OK;
}

dvg_status dvg_l2_device(dvg_context* ctx, const float* image, const float* target, uint64_t n, float* d_render,
                         float* loss) {
    if (!ctx || !image || !target || !d_render) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    if (loss) CK(cudaMemsetAsync(loss, 0, sizeof(float), ctx->stream));
    if (n == 0) return DVG_OK;
    Prof prof_(ctx, "l2_loss");
    ctx->launches += launch_l2(image, target, (size_t)n, d_render, loss, ctx->stream);
    CK(cudaGetLastError());
    return DVG_OK;
}

dvg_status dvg_shard_backward(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                              const dvg_backward_options* bopts, const dvg_shard* shard, const float* d_render,
                              const float* wsum, dvg_grads* grads) {
    dvg_status st = check_backward_args(ctx, scene, opts, nullptr, grads);
    if (st == DVG_OK) st = check_shard(scene, shard);
    if (st != DVG_OK) return st;
    if (!d_render || !wsum) return fail(DVG_ERR_INVALID_ARGUMENT, "null d_render or weights");
    CK(cudaSetDevice(ctx->device));
    GradPtrs G = grads_from_user(grads);
    if (!(bopts && bopts->compute_translation)) G.d_translation = nullptr;
    if (!scene->dev.bg_image) G.d_background_image = nullptr;
    st = zero_grads(ctx, scene, G);
    if (st != DVG_OK) return st;
    // The codes are laid out by the tuning's slot count and sample layout: a
    // dvg_scene_set_tuning between the two calls makes them unusable.
    const bool frag = ctx->shard_frag && ctx->shard_scene == scene && ctx->shard_gen == ctx->gen &&
                      ctx->shard_t0 == shard->tile_begin && ctx->shard_t1 == shard->tile_end &&
                      std::memcmp(&ctx->shard_opts, opts, sizeof(dvg_render_options)) == 0 &&
                      std::memcmp(&ctx->shard_tune, &scene->tune, sizeof(dvg_tuning)) == 0;
    return backward_core(ctx, scene, opts, bopts, d_render, nullptr, G, true, frag, shard, wsum);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Render without any device allocation.
//
// For callers that cannot call cudaMalloc while they render: a host application
// that hands this library a fixed device-memory budget up front, a plugin that
// runs inside another framework's frame loop where allocation is not allowed,
// or code that must not hit the allocator's implicit synchronisation.  The
// filtered-splat accumulators (4 colour floats + 1 weight float per pixel)
// live in one file-scope device array instead of the context's grow-only
// scratch, so a call only launches kernels and clears that array.
//
// Limits and sharing:
//   * at most kNoAllocMaxPixels (512*512) pixels per canvas; larger canvases are
//     rejected with DVG_ERR_INVALID_ARGUMENT before anything is launched;
//   * every GPU that loads this library holds the array (5 MiB) until exit;
//   * all calls on a device share the one array and it keeps the last call's
//     contents: each call clears it first, and calls whose work overlaps on the
//     GPU (different streams or contexts at the same time) race on it.
// The array's device address is looked up once per device, by the first call
// on that device (with the device current); make that first call before any
// stream capture begins.
namespace {
constexpr size_t kNoAllocMaxPixels = 512 * 512;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocMaxPixels * 5];
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

dvg_status noalloc_scratch(int device, float** out) {
    if (device < 0 || device >= kNoAllocMaxDevices)
        return fail(DVG_ERR_INVALID_ARGUMENT, "device ordinal beyond the no-allocation table");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[device] = p;
    }
    *out = static_cast<float*>(g_noalloc_ptr[device]);
    return DVG_OK;
}
}  // namespace

extern "C" dvg_status dvg_render_device_noalloc(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                                float* out_rgba) {
    if (!ctx || !scene || !out_rgba) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    const DevScene& S = scene->dev;
    const size_t npix = (size_t)S.width * S.height;
    if (npix == 0) return DVG_OK;
    if (npix > kNoAllocMaxPixels)
        return fail(DVG_ERR_INVALID_ARGUMENT,
                    "canvas of " + std::to_string(npix) + " pixels exceeds the no-allocation limit of " +
                        std::to_string(kNoAllocMaxPixels) + " pixels (512x512); use dvg_render_device");
    float* scratch = nullptr;
    st = noalloc_scratch(ctx->device, &scratch);
    if (st != DVG_OK) return st;
    if (S.num_groups == 0) {
        ctx->launches += launch_fill_background(S, out_rgba, ctx->stream);
        CK(cudaGetLastError());
        return DVG_OK;
    }
    float* accum = scratch;            // 4 floats per pixel (float4 aligned: 256-byte base)
    float* wsum = scratch + 4 * npix;  // 1 float per pixel
    CK(cudaMemsetAsync(scratch, 0, 5 * npix * sizeof(float), ctx->stream));
    const SampleParams sp = sample_params(opts, scene->tune);
    if (opts->use_prefiltering)
        ctx->launches += launch_forward_prefilter(S, sp, accum, wsum, ctx->status, ctx->stream);
    else
        ctx->launches += launch_forward(S, sp, accum, wsum, ctx->status, ctx->stream);
    ctx->launches += launch_resolve(S, accum, wsum, out_rgba, ctx->stream);
    CK(cudaGetLastError());
    return DVG_OK;
}

// ---------------------------------------------------------------------------
// Batches: many uploaded scenes stepped together (forward + L2 + backward), one
// kernel launch per stage for all scenes, optionally replayed as one CUDA graph.
struct dvg_batch {
    dvg_context* ctx = nullptr;
    std::vector<dvg_scene*> scenes;
    dvg_render_options opts{};
    dvg_backward_options bopts{};
    std::vector<BatchEntry> host_entries;
    std::vector<size_t> pix_off;      // float offset of each scene's 4-channel image region
    std::vector<size_t> wpix_off;     // float offset of each scene's 1-channel region
    std::vector<size_t> grad_base;    // float offset of each scene's gradient block
    size_t total_pix4 = 0, total_pix = 0, total_grads = 0, max_pixels = 0;
    int items = 0, total_tiles = 0, max_ri = 0;
    uint64_t total_bsamples = 0;
    DevBuf entries, work, queue, accum, wsum, image, target, d_render, loss, grads, bsamples, bkey, border, bcounts;
    DevBuf frag;  // per-scene fragment caches (forward -> interior)
    bool any_styled = false;  // some scene strokes with non-round joins or caps
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t steps = 0;
    dvg_tuning tune{1, 4, 16, 0, 0};  // launch shape (dvg_batch_autotune)
    // on-device optimisation step (dvg_batch_set_adam)
    bool adam = false;
    AdamParams ap{};
    DevBuf refit, adam_state, sort_ids, sort_keys, opt_step;
    int max_params = 0, max_paths = 0, max_groups = 0;
};

namespace {
dvg_status batch_enqueue(dvg_batch* b) {
    dvg_context* ctx = b->ctx;
    const int n = (int)b->scenes.size();
    const BatchEntry* B = b->entries.as<BatchEntry>();
    CK(cudaMemsetAsync(b->accum.ptr, 0, b->total_pix4 * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(b->wsum.ptr, 0, b->total_pix * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(b->loss.ptr, 0, (size_t)n * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(b->grads.ptr, 0, b->total_grads * sizeof(float), ctx->stream));
    const bool pre = b->opts.use_prefiltering != 0;
    int* queue = nullptr;  // persistent CTAs: three zeroed item counters (forward, 2 interior kernels)
    if (b->tune.work_queue) {
        CK(b->queue.reserve(4 * sizeof(int)));
        CK(cudaMemsetAsync(b->queue.ptr, 0, 4 * sizeof(int), ctx->stream));
        queue = b->queue.as<int>();
    }
    if (pre)
        ctx->launches += launch_forward_prefilter_batch(B, b->work.as<int2>(), b->items, queue, b->max_ri,
                                                        ctx->status, ctx->stream);
    else
        ctx->launches += launch_forward_batch(B, b->work.as<int2>(), b->items, queue, b->max_ri,
                                              (int)b->tune.forward_occupancy, ctx->stream);
    ctx->launches += launch_pixels_batch(B, n, b->max_pixels, 0, ctx->stream);
    ctx->launches += launch_pixels_batch(B, n, b->max_pixels, 1, ctx->stream);
    if (pre)
        ctx->launches += launch_interior_prefilter_batch(B, b->work.as<int2>(), b->items, queue ? queue + 1 : nullptr,
                                                         ctx->status, ctx->stream);
    else
        ctx->launches += launch_interior_batch(B, b->work.as<int2>(), b->items, queue ? queue + 1 : nullptr,
                                               ctx->status, ctx->stream);
    if (!pre)
        ctx->launches += launch_boundary_batch(B, n, b->total_bsamples, b->total_tiles, (int)b->tune.boundary_cell,
                                               b->any_styled,
                                               b->bsamples.as<BSample>(),
                                               b->bkey.as<int>(), b->bcounts.as<int>(), b->border.as<int>(),
                                               ctx->stream);
    ctx->launches += launch_pixels_batch(B, n, b->max_pixels, 2, ctx->stream);
    if (b->adam) {
        BatchEntry* Bm = b->entries.as<BatchEntry>();
        const RefitEntry* R = b->refit.as<RefitEntry>();
        ctx->launches += launch_adam_batch(Bm, R, n, b->max_params, b->ap, b->opt_step.as<int>(), ctx->stream);
        ctx->launches += launch_refit_batch(Bm, R, n, b->max_paths, b->max_groups, ctx->status, ctx->stream);
        for (dvg_scene* sc : b->scenes) {
            int* counts = sc->tiles.as<int>();
            int* offsets = counts + sc->dev.tiles_x * sc->dev.tiles_y;
            ctx->launches += launch_binning(sc->dev, sc->g_bbox, counts, offsets, nullptr, ctx->stream);
            ctx->launches += launch_binning(sc->dev, sc->g_bbox, counts, offsets, sc->entries.as<int>(), ctx->stream);
        }
    }
    CK(cudaGetLastError());
    return DVG_OK;
}
// Applies b->tune to the host entries: warp layout, and one fragment cache per scene
// inside b->frag (none when prefiltering or with zero slots).
dvg_status batch_apply_tuning(dvg_batch* b) {
    const int slots = b->opts.use_prefiltering ? 0 : (int)b->tune.fragment_slots;
    std::vector<size_t> off;
    size_t total = 0;
    for (const BatchEntry& e : b->host_entries) {
        off.push_back(total);
        total += (frag_cache_bytes(e.S.tiles_x * e.S.tiles_y, e.sp.sxn * e.sp.syn, slots) + 255) & ~(size_t)255;
    }
    if (slots > 0) CK(b->frag.reserve(total));
    for (size_t i = 0; i < b->host_entries.size(); ++i) {
        BatchEntry& e = b->host_entries[i];
        e.sp.layout = (int)b->tune.sample_layout;
        e.sp.fwd_occ = (int)b->tune.forward_occupancy;
        e.sp.frag = nullptr;
        e.sp.frag_n = nullptr;
        e.sp.frag_slots = 0;
        if (slots > 0) attach_frag(e.sp, b->frag.as<char>() + off[i], e.S.tiles_x * e.S.tiles_y, slots);
    }
    return DVG_OK;
}
void batch_drop_graph(dvg_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}
}  // namespace

extern "C" dvg_status dvg_batch_create(dvg_context* ctx, dvg_scene* const* scenes, uint32_t count,
                                       const dvg_render_options* opts, const dvg_backward_options* bopts,
                                       dvg_batch** out) {
    if (!ctx || !scenes || !opts || !out || count == 0) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    std::unique_ptr<dvg_batch> b(new dvg_batch());
    b->ctx = ctx;
    b->opts = *opts;
    if (bopts) b->bopts = *bopts;
    else {
        b->bopts.boundary_seed_from_options = 1;
    }
    const SampleParams sp = sample_params(opts, dvg_tuning{1, 4, 16, 0, 0});
    // Work items (scene, tile + tiles * sub-sample round), one CTA each, listed heaviest
    // first: the hardware hands out CTAs in list order as SMs free up, so the longest
    // items start first and the stage's tail is made of short ones.  Weight: the groups
    // binned to the item's tile + 1 (its sampling and splat).
    struct Item {
        int weight, scene, local;
    };
    std::vector<Item> work;
    for (uint32_t i = 0; i < count; ++i) {
        dvg_scene* sc = scenes[i];
        if (!sc || sc->ctx != ctx) return fail(DVG_ERR_INVALID_ARGUMENT, "batch scene is null or from another context");
        const DevScene& S = sc->dev;
        const size_t npix = (size_t)S.width * S.height;
        if (npix == 0 || S.num_groups == 0)
            return fail(DVG_ERR_INVALID_ARGUMENT, "batch scenes need a non-empty canvas and at least one group");
        b->scenes.push_back(sc);
        b->any_styled = b->any_styled || S.styled;
        b->pix_off.push_back(b->total_pix4);
        b->wpix_off.push_back(b->total_pix);
        b->total_pix4 += (npix * 4 + 63) & ~(size_t)63;
        b->total_pix += (npix + 63) & ~(size_t)63;
        b->max_pixels = std::max(b->max_pixels, npix);
        b->grad_base.push_back(b->total_grads);
        b->total_grads += (sc->grad_floats + 63) & ~(size_t)63;
        b->max_ri = std::max(b->max_ri, S.filter_ri);
        BatchEntry e{};
        e.S = S;
        e.sp = sp;
        e.item_off = b->items;
        const int tiles = S.tiles_x * S.tiles_y;
        e.tile_off = b->total_tiles;
        const uint64_t spp = (uint64_t)sp.sxn * sp.syn;
        e.nb = b->bopts.boundary_samples ? b->bopts.boundary_samples : (uint64_t)npix * spp;
        // (scenes without boundary tables draw no samples: the generator checks the flag,
        // which the on-device optimisation step may turn on or off)
        e.b_off = b->total_bsamples;
        e.bseed = b->bopts.boundary_seed_from_options ? opts->seed : b->bopts.boundary_seed;
        e.rng = (int)b->bopts.rng;
        e.bscale = (float)((double)e.nb / (double)((uint64_t)npix * spp));
        const int items = tiles * (int)spp;
        std::vector<int> off(tiles + 1, 0);
        CK(cudaMemcpyAsync(off.data(), S.tile_offsets, (tiles + 1) * sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (int k = 0; k < items; ++k) work.push_back(Item{off[k % tiles + 1] - off[k % tiles] + 1, (int)i, k});
        b->items += items;
        b->total_tiles += tiles;
        b->total_bsamples += e.nb;
        b->host_entries.push_back(e);
    }
    CK(b->accum.reserve(b->total_pix4 * sizeof(float)));
    CK(b->image.reserve(b->total_pix4 * sizeof(float)));
    CK(b->target.reserve(b->total_pix4 * sizeof(float)));
    CK(b->d_render.reserve(b->total_pix4 * sizeof(float)));
    CK(b->wsum.reserve(b->total_pix * sizeof(float)));
    CK(b->loss.reserve(count * sizeof(float)));
    CK(b->grads.reserve(std::max<size_t>(b->total_grads, 64) * sizeof(float)));
    std::stable_sort(work.begin(), work.end(), [](const Item& x, const Item& y) { return x.weight > y.weight; });
    std::vector<int2> work2(work.size());
    for (size_t k = 0; k < work.size(); ++k) work2[k] = make_int2(work[k].scene, work[k].local);
    CK(b->work.reserve(work2.size() * sizeof(int2)));
    const uint64_t nbs = std::max<uint64_t>(b->total_bsamples, 1);
    CK(b->bsamples.reserve(nbs * sizeof(BSample)));
    CK(b->bkey.reserve(nbs * sizeof(int)));
    CK(b->border.reserve(nbs * sizeof(int)));
    CK(b->bcounts.reserve(bnd_count_ints((size_t)b->total_tiles) * sizeof(int)));
    CK(cudaMemsetAsync(b->target.ptr, 0, b->total_pix4 * sizeof(float), ctx->stream));
    float* acc = b->accum.as<float>();
    float* img = b->image.as<float>();
    float* tgt = b->target.as<float>();
    float* dr = b->d_render.as<float>();
    float* ws = b->wsum.as<float>();
    float* gb = b->grads.as<float>();
    for (uint32_t i = 0; i < count; ++i) {
        BatchEntry& e = b->host_entries[i];
        dvg_scene* sc = b->scenes[i];
        e.accum = acc + b->pix_off[i];
        e.image = img + b->pix_off[i];
        e.target = tgt + b->pix_off[i];
        e.d_render = dr + b->pix_off[i];
        e.wsum = ws + b->wpix_off[i];
        e.loss = b->loss.as<float>() + i;
        float* g = gb + b->grad_base[i];
        e.G.d_shape_params = g + sc->grad_off[0];
        e.G.d_shape_transform = g + sc->grad_off[1];
        e.G.d_shape_stroke_width = g + sc->grad_off[2];
        e.G.d_points = g + sc->grad_off[3];
        e.G.d_thickness = g + sc->grad_off[4];
        e.G.d_group_transform = g + sc->grad_off[5];
        e.G.d_paint_params = g + sc->grad_off[6];
        e.G.d_stop_offsets = g + sc->grad_off[7];
        e.G.d_stop_colors = g + sc->grad_off[8];
        e.G.d_filter_radius = g + sc->grad_off[9];
        e.G.d_background = g + sc->grad_off[10];
        e.G.d_background_image = nullptr;
        e.G.d_translation = nullptr;
    }
    st = batch_apply_tuning(b.get());
    if (st != DVG_OK) return st;
    CK(b->entries.reserve(count * sizeof(BatchEntry)));
    CK(cudaMemcpyAsync(b->entries.ptr, b->host_entries.data(), count * sizeof(BatchEntry), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaMemcpyAsync(b->work.ptr, work2.data(), work2.size() * sizeof(int2), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *out = b.release();
    return DVG_OK;
}

extern "C" void dvg_batch_destroy(dvg_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    batch_drop_graph(b);
    delete b;
}

extern "C" dvg_status dvg_batch_buffers(dvg_batch* b, uint32_t index, float** image, float** target,
                                        dvg_grads* grads) {
    if (!b || index >= b->scenes.size()) return fail(DVG_ERR_INVALID_ARGUMENT, "batch index out of range");
    const BatchEntry& e = b->host_entries[index];
    if (image) *image = e.image;
    if (target) *target = const_cast<float*>(e.target);
    if (grads) {
        grads->d_shape_params = e.G.d_shape_params;
        grads->d_shape_transform = e.G.d_shape_transform;
        grads->d_shape_stroke_width = e.G.d_shape_stroke_width;
        grads->d_points = e.G.d_points;
        grads->d_thickness = e.G.d_thickness;
        grads->d_group_transform = e.G.d_group_transform;
        grads->d_paint_params = e.G.d_paint_params;
        grads->d_stop_offsets = e.G.d_stop_offsets;
        grads->d_stop_colors = e.G.d_stop_colors;
        grads->d_filter_radius = e.G.d_filter_radius;
        grads->d_background = e.G.d_background;
        grads->d_background_image = nullptr;
        grads->d_translation = nullptr;
    }
    return DVG_OK;
}

extern "C" dvg_status dvg_batch_step(dvg_batch* b, int use_graph) {
    if (!b) return fail(DVG_ERR_INVALID_ARGUMENT, "null batch");
    dvg_context* ctx = b->ctx;
    CK(cudaSetDevice(ctx->device));
    if (!use_graph) {
        b->steps++;
        return batch_enqueue(b);
    }
    if (!b->exec) {
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        dvg_status st = batch_enqueue(b);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (st != DVG_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        b->graph = g;
        CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    CK(cudaGraphLaunch(b->exec, ctx->stream));
    b->steps++;
    return DVG_OK;
}

extern "C" dvg_status dvg_batch_losses(dvg_batch* b, float* host_losses) {
    if (!b || !host_losses) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_context* ctx = b->ctx;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(host_losses, b->loss.ptr, b->scenes.size() * sizeof(float), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

extern "C" dvg_status dvg_batch_set_adam(dvg_batch* b, const dvg_adam_options* o) {
    if (!b) return fail(DVG_ERR_INVALID_ARGUMENT, "null batch");
    dvg_context* ctx = b->ctx;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    batch_drop_graph(b);
    if (!o) {
        b->adam = false;
        return DVG_OK;
    }
    if (!(std::isfinite(o->lr) && o->lr >= 0.0f && o->beta1 >= 0.0f && o->beta1 < 1.0f && o->beta2 >= 0.0f &&
          o->beta2 < 1.0f && std::isfinite(o->eps) && o->eps >= 0.0f) ||
        (o->params & ~(uint32_t)(DVG_OPT_POINTS | DVG_OPT_PAINTS)) || !o->params)
        return fail(DVG_ERR_INVALID_ARGUMENT, "invalid Adam options");
    const int n = (int)b->scenes.size();
    AdamParams ap{o->lr, o->beta1, o->beta2, o->eps, (o->params & DVG_OPT_POINTS) ? 1 : 0,
                  (o->params & DVG_OPT_PAINTS) ? 1 : 0};
    // Tile lists must hold any binning the moved geometry can produce: every group in
    // every tile at worst.
    for (int i = 0; i < n; ++i) {
        dvg_scene* sc = b->scenes[i];
        const size_t tiles = (size_t)sc->dev.tiles_x * sc->dev.tiles_y;
        const size_t need = std::max<size_t>(tiles * (size_t)std::max(sc->dev.num_groups, 1), 1);
        if (need > ((size_t)1 << 28))
            return fail(DVG_ERR_DEVICE_LIMIT, "tile lists of an optimised scene would exceed 2^28 entries");
        if (sc->entries.bytes < need * sizeof(int)) {
            CK(sc->entries.reserve(need * sizeof(int)));
            sc->dev.tile_entries = sc->entries.as<int>();
            int* counts = sc->tiles.as<int>();
            int* offsets = counts + tiles;
            ctx->launches += launch_binning(sc->dev, sc->g_bbox, counts, offsets, nullptr, ctx->stream);
            ctx->launches += launch_binning(sc->dev, sc->g_bbox, counts, offsets, sc->entries.as<int>(), ctx->stream);
            CK(cudaGetLastError());
        }
        b->host_entries[i].S.tile_entries = sc->dev.tile_entries;
    }
    // Adam moments and sort scratch, one block per scene.
    std::vector<size_t> st_off(n), so_off(n);
    size_t st_total = 0, so_total = 0;
    int max_params = 0, max_paths = 0, max_groups = 0;
    for (int i = 0; i < n; ++i) {
        const HostScene& h = b->scenes[i]->host;
        const size_t np = ap.points ? 2 * (size_t)h.total_points : 0;
        const size_t nq = ap.paints ? 4 * (size_t)h.num_paints : 0;
        st_off[i] = st_total;
        st_total += 2 * ((np + nq + 63) & ~(size_t)63);
        const size_t sort_n = std::max(h.seg_meta.size() / 4, h.g_shape_list.size());
        so_off[i] = so_total;
        so_total += 2 * ((sort_n + 63) & ~(size_t)63);
        max_params = std::max(max_params, (int)(np + nq));
        max_paths = std::max(max_paths, (int)h.num_paths);
        max_groups = std::max(max_groups, (int)h.num_groups);
    }
    CK(b->adam_state.reserve(std::max<size_t>(st_total, 64) * sizeof(float)));
    CK(b->sort_ids.reserve(std::max<size_t>(so_total, 64) * sizeof(int)));
    CK(b->sort_keys.reserve(std::max<size_t>(so_total, 64) * sizeof(float)));
    CK(b->opt_step.reserve(sizeof(int)));
    CK(cudaMemsetAsync(b->adam_state.ptr, 0, std::max<size_t>(st_total, 64) * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(b->opt_step.ptr, 0, sizeof(int), ctx->stream));
    std::vector<RefitEntry> re(n);
    for (int i = 0; i < n; ++i) {
        dvg_scene* sc = b->scenes[i];
        const HostScene& h = sc->host;
        const size_t np = ap.points ? 2 * (size_t)h.total_points : 0;
        const size_t nq = ap.paints ? 4 * (size_t)h.num_paints : 0;
        const size_t half = (np + nq + 63) & ~(size_t)63;
        float* base = b->adam_state.as<float>() + st_off[i];
        RefitEntry& r = re[i];
        r.m_points = base;
        r.v_points = base + half;
        r.m_paints = base + np;
        r.v_paints = base + half + np;
        r.sort_n = (int)std::max(h.seg_meta.size() / 4, h.g_shape_list.size());
        r.sort_ids = b->sort_ids.as<int>() + so_off[i];
        r.sort_keys = b->sort_keys.as<float>() + so_off[i];
        r.n_points = (int)h.total_points;
        r.n_paints = (int)h.num_paints;
        r.g_bbox = const_cast<float4*>(sc->g_bbox);
    }
    CK(b->refit.reserve(n * sizeof(RefitEntry)));
    CK(cudaMemcpyAsync(b->refit.ptr, re.data(), n * sizeof(RefitEntry), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b->entries.ptr, b->host_entries.data(), n * sizeof(BatchEntry), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    b->ap = ap;
    b->max_params = max_params;
    b->max_paths = max_paths;
    b->max_groups = max_groups;
    b->adam = true;
    return DVG_OK;
}

extern "C" dvg_status dvg_batch_scene_params(dvg_batch* b, uint32_t index, float* host_points,
                                             float* host_paint_params) {
    if (!b || index >= b->scenes.size()) return fail(DVG_ERR_INVALID_ARGUMENT, "batch index out of range");
    dvg_context* ctx = b->ctx;
    CK(cudaSetDevice(ctx->device));
    dvg_scene* sc = b->scenes[index];
    const HostScene& h = sc->host;
    if (host_points && h.total_points)
        CK(cudaMemcpyAsync(host_points, sc->dev.points, 2 * (size_t)h.total_points * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->stream));
    if (host_paint_params && h.num_paints)
        CK(cudaMemcpyAsync(host_paint_params, sc->dev.paint_params, 4 * (size_t)h.num_paints * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->stream));
    int ok = sc->dev.boundary_ok;
    const BatchEntry* E = b->entries.as<BatchEntry>() + index;
    CK(cudaMemcpyAsync(&ok, &E->S.boundary_ok, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    sc->dev.boundary_ok = ok;
    b->host_entries[index].S.boundary_ok = ok;
    return check_status(ctx);
}

extern "C" dvg_status dvg_scene_digest(dvg_context* ctx, dvg_scene* sc, uint64_t* digest) {
    if (!ctx || !sc || !digest) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    const int tiles = sc->dev.tiles_x * sc->dev.tiles_y;
    std::vector<char> arena(sc->arena_bytes);
    std::vector<int> tl(tiles > 0 ? 2 * (size_t)tiles + 1 : 0);
    if (!arena.empty())
        CK(cudaMemcpyAsync(arena.data(), sc->arena.ptr, arena.size(), cudaMemcpyDeviceToHost, ctx->stream));
    if (!tl.empty())
        CK(cudaMemcpyAsync(tl.data(), sc->tiles.ptr, tl.size() * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<int> entries(tiles > 0 ? (size_t)std::max(tl[2 * (size_t)tiles], 0) : 0);
    if (!entries.empty()) {
        CK(cudaMemcpyAsync(entries.data(), sc->entries.ptr, entries.size() * sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    uint64_t h = 1469598103934665603ull;  // FNV-1a, 64 bit
    auto mix = [&h](const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) {
            h ^= c[i];
            h *= 1099511628211ull;
        }
    };
    mix(arena.data(), arena.size());
    if (tiles > 0) mix(tl.data() + tiles, ((size_t)tiles + 1) * sizeof(int));  // offsets (counts are scratch)
    mix(entries.data(), entries.size() * sizeof(int));
    int flags[1] = {sc->dev.boundary_ok};
    mix(flags, sizeof(flags));
    *digest = h;
    return DVG_OK;
}

// ------------------------------------------------------------------ signed distance field
extern "C" dvg_status dvg_render_sdf_device(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                            float* out) {
    if (!ctx || !scene || !out) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    const DevScene& S = scene->dev;
    const size_t npix = (size_t)S.width * S.height;
    if (npix == 0) return DVG_OK;
    if (S.num_groups == 0) {
        CK(cudaMemsetAsync(out, 0, npix * sizeof(float), ctx->stream));
        return DVG_OK;
    }
    {
        Prof prof_(ctx, "render_sdf");
        ctx->launches += launch_render_sdf(S, sample_params(opts, dvg_tuning{1, 4, 16, 0, 0}), out, ctx->status, ctx->stream);
    }
    CK(cudaGetLastError());
    return DVG_OK;
}

extern "C" dvg_status dvg_render_sdf_host(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                          float* out) {
    if (!ctx || !scene || !out) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    const size_t npix = (size_t)scene->dev.width * scene->dev.height;
    if (npix == 0) return check_options(opts);
    CK(ctx->sdf.reserve(npix * sizeof(float)));
    dvg_status st = dvg_render_sdf_device(ctx, scene, opts, ctx->sdf.as<float>());
    if (st != DVG_OK) return st;
    CK(cudaMemcpyAsync(out, ctx->sdf.ptr, npix * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

extern "C" dvg_status dvg_render_sdf(dvg_context* ctx, const dvg_scene_desc* desc, const dvg_render_options* opts,
                                     float* out) {
    if (!ctx || !desc || !out) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    dvg_scene* sc = nullptr;
    st = dvg_scene_upload(ctx, desc, &sc);
    if (st != DVG_OK) return st;
    st = dvg_render_sdf_host(ctx, sc, opts, out);
    dvg_scene_destroy(sc);
    return st;
}

extern "C" dvg_status dvg_eval_positions_device(dvg_context* ctx, dvg_scene* scene, const float* positions,
                                                uint64_t count, float* out) {
    if (!ctx || !scene || (count && (!positions || !out))) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    if (count == 0) return DVG_OK;
    if (scene->dev.num_groups == 0) {
        CK(cudaMemsetAsync(out, 0, count * sizeof(float), ctx->stream));
        return DVG_OK;
    }
    {
        Prof prof_(ctx, "eval_positions");
        ctx->launches += launch_eval_positions(scene->dev, reinterpret_cast<const float2*>(positions), count, out,
                                               ctx->status, ctx->stream);
    }
    CK(cudaGetLastError());
    return DVG_OK;
}

extern "C" dvg_status dvg_eval_positions_host(dvg_context* ctx, dvg_scene* scene, const float* positions,
                                              uint64_t count, float* out) {
    if (!ctx || !scene || (count && (!positions || !out))) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    if (count == 0) return DVG_OK;
    CK(ctx->positions.reserve(count * 2 * sizeof(float)));
    CK(ctx->dvalues.reserve(count * sizeof(float)));
    CK(cudaMemcpyAsync(ctx->positions.ptr, positions, count * 2 * sizeof(float), cudaMemcpyHostToDevice,
                       ctx->stream));
    dvg_status st = dvg_eval_positions_device(ctx, scene, ctx->positions.as<float>(), count, ctx->dvalues.as<float>());
    if (st != DVG_OK) return st;
    CK(cudaMemcpyAsync(out, ctx->dvalues.ptr, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

extern "C" dvg_status dvg_eval_positions(dvg_context* ctx, const dvg_scene_desc* desc, const float* positions,
                                         uint64_t count, float* out) {
    if (!ctx || !desc) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    if (count == 0) return DVG_OK;
    dvg_scene* sc = nullptr;
    dvg_status st = dvg_scene_upload(ctx, desc, &sc);
    if (st != DVG_OK) return st;
    st = dvg_eval_positions_host(ctx, sc, positions, count, out);
    dvg_scene_destroy(sc);
    return st;
}

extern "C" dvg_status dvg_eval_positions_backward_device(dvg_context* ctx, dvg_scene* scene,
                                                         const dvg_backward_options* bopts, const float* positions,
                                                         uint64_t count, const float* d_values, dvg_grads* grads) {
    if (!ctx || !scene || !grads || (count && (!positions || !d_values)))
        return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    GradPtrs G = grads_from_user(grads);
    const bool tr = bopts && bopts->compute_translation && G.d_translation;
    if (!tr) G.d_translation = nullptr;
    G.d_background_image = nullptr;
    dvg_status st = zero_grads(ctx, scene, grads_from_user(grads));
    if (st != DVG_OK) return st;
    if (count == 0 || scene->dev.num_groups == 0) return DVG_OK;
    {
        Prof prof_(ctx, "positions_backward");
        ctx->launches += launch_positions_backward(scene->dev, reinterpret_cast<const float2*>(positions), count,
                                                   d_values, G, tr, ctx->status, ctx->stream);
    }
    CK(cudaGetLastError());
    return DVG_OK;
}

extern "C" dvg_status dvg_eval_positions_backward_host(dvg_context* ctx, dvg_scene* scene,
                                                       const dvg_backward_options* bopts, const float* positions,
                                                       uint64_t count, const float* d_values, dvg_grads* grads) {
    if (!ctx || !scene || !grads || (count && (!positions || !d_values)))
        return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    const HostScene& h = scene->host;
    const size_t npix = (size_t)h.width * h.height;
    GradPtrs G = device_grads(scene);
    CK(cudaMemsetAsync(scene->grads.ptr, 0, scene->grad_floats * sizeof(float), ctx->stream));
    const bool want_tr = bopts && bopts->compute_translation && grads->d_translation && npix;
    G.d_background_image = nullptr;
    G.d_translation = nullptr;
    if (want_tr) {
        CK(ctx->trans_grad.reserve(npix * 2 * sizeof(float)));
        CK(cudaMemsetAsync(ctx->trans_grad.ptr, 0, npix * 2 * sizeof(float), ctx->stream));
        G.d_translation = ctx->trans_grad.as<float>();
    }
    if (count && scene->dev.num_groups > 0) {
        CK(ctx->positions.reserve(count * 2 * sizeof(float)));
        CK(ctx->dvalues.reserve(count * sizeof(float)));
        CK(cudaMemcpyAsync(ctx->positions.ptr, positions, count * 2 * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(cudaMemcpyAsync(ctx->dvalues.ptr, d_values, count * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        Prof prof_(ctx, "positions_backward");
        ctx->launches += launch_positions_backward(scene->dev, ctx->positions.as<float2>(), count,
                                                   ctx->dvalues.as<float>(), G, want_tr, ctx->status, ctx->stream);
        CK(cudaGetLastError());
    }
    struct Part {
        float* dst;
        const float* src;
        size_t n;
    } parts[] = {{grads->d_shape_params, G.d_shape_params, 4 * (size_t)h.num_shapes},
                 {grads->d_shape_transform, G.d_shape_transform, 9 * (size_t)h.num_shapes},
                 {grads->d_shape_stroke_width, G.d_shape_stroke_width, h.num_shapes},
                 {grads->d_points, G.d_points, 2 * (size_t)h.total_points},
                 {grads->d_thickness, G.d_thickness, h.total_points},
                 {grads->d_group_transform, G.d_group_transform, 9 * (size_t)h.num_groups},
                 {grads->d_paint_params, G.d_paint_params, 4 * (size_t)h.num_paints},
                 {grads->d_stop_offsets, G.d_stop_offsets, h.total_stops},
                 {grads->d_stop_colors, G.d_stop_colors, 4 * (size_t)h.total_stops},
                 {grads->d_filter_radius, G.d_filter_radius, 1},
                 {grads->d_background, G.d_background, 4}};
    for (auto& p : parts)
        if (p.dst && p.n) CK(cudaMemcpyAsync(p.dst, p.src, p.n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (grads->d_background_image) std::memset(grads->d_background_image, 0, npix * 4 * sizeof(float));
    if (grads->d_translation) {
        if (want_tr)
            CK(cudaMemcpyAsync(grads->d_translation, G.d_translation, npix * 2 * sizeof(float),
                               cudaMemcpyDeviceToHost, ctx->stream));
        else
            std::memset(grads->d_translation, 0, npix * 2 * sizeof(float));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

extern "C" dvg_status dvg_eval_positions_backward(dvg_context* ctx, const dvg_scene_desc* desc,
                                                  const dvg_backward_options* bopts, const float* positions,
                                                  uint64_t count, const float* d_values, dvg_grads* grads) {
    if (!ctx || !desc || !grads) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_scene* sc = nullptr;
    dvg_status st = dvg_scene_upload(ctx, desc, &sc);
    if (st != DVG_OK) return st;
    st = dvg_eval_positions_backward_host(ctx, sc, bopts, positions, count, d_values, grads);
    dvg_scene_destroy(sc);
    return st;
}

extern "C" dvg_status dvg_lbvh_build(dvg_context* ctx, const float* boxes, uint32_t count, uint64_t* keys_out,
                                     int32_t* children_out, float* bounds_out) {
    if (!ctx || (count && !boxes)) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    if (count > (1u << 24)) return fail(DVG_ERR_INVALID_ARGUMENT, "more than 2^24 boxes");
    CK(cudaSetDevice(ctx->device));
    if (count == 0) return DVG_OK;
    const int n = (int)count;
    const size_t padded = (size_t)lbvh_padded(n);
    DevBuf buf;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = (off + 255) & ~(size_t)255;
        off = o + std::max<size_t>(bytes, 16);
        return o;
    };
    const size_t o_box = take(sizeof(float4) * n), o_keys = take(padded * 8),
                 o_child = take(sizeof(int2) * (size_t)std::max(n - 1, 0)), o_par = take(sizeof(int) * (2 * n - 1)),
                 o_flag = take(sizeof(int) * (size_t)std::max(n - 1, 0)), o_bnd = take(sizeof(float4) * (2 * n - 1)),
                 o_leaf = take(sizeof(int) * n), o_ext = take(sizeof(float4));
    CK(buf.reserve(off));
    char* b = buf.as<char>();
    LbvhBufs L{(uint64_t*)(b + o_keys), (int2*)(b + o_child), (int*)(b + o_par), (int*)(b + o_flag),
               (float4*)(b + o_bnd), (int*)(b + o_leaf), (float4*)(b + o_ext)};
    CK(cudaMemcpyAsync(b + o_box, boxes, sizeof(float4) * n, cudaMemcpyHostToDevice, ctx->stream));
    ctx->launches += launch_lbvh_build((const float4*)(b + o_box), n, nullptr, L, ctx->stream);
    CK(cudaGetLastError());
    if (keys_out) CK(cudaMemcpyAsync(keys_out, L.keys, 8 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    if (children_out && n > 1)
        CK(cudaMemcpyAsync(children_out, L.children, sizeof(int2) * (size_t)(n - 1), cudaMemcpyDeviceToHost,
                           ctx->stream));
    if (bounds_out)
        CK(cudaMemcpyAsync(bounds_out, L.bounds, sizeof(float4) * (size_t)(2 * n - 1), cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return DVG_OK;
}

// ------------------------------------------------------------------ launch-shape tuning
namespace {
bool tuning_valid(const dvg_tuning* t) {
    return t && t->sample_layout <= 1 &&
           (t->boundary_cell == 2 || t->boundary_cell == 4 || t->boundary_cell == 8 || t->boundary_cell == 16) &&
           t->fragment_slots <= (uint32_t)FRAG_MAX_SLOTS && t->work_queue <= 1 &&
           t->forward_occupancy <= 2;
}
// The candidates: both warp layouts with the default cell and cache, then every cell
// with the better layout (the boundary pass does not depend on the layout), then the
// fragment-cache sizes (`try_slots`: only where the cache is used, non-prefiltered),
// then persistent CTAs for the batch stages (`try_queue`), then the forward kernel at
// 3 and at 2 CTAs per SM.
template <typename Apply, typename Run>
dvg_status autotune_loop(dvg_context* ctx, dvg_tuning* tune, bool try_slots, Apply apply, Run run,
                         bool try_queue = false) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // a candidate's time: the median of three timed runs after one warm run
    auto time_of = [&](dvg_tuning t, float* ms) -> dvg_status {
        *tune = t;
        dvg_status st = apply();
        if (st != DVG_OK) return st;
        st = run();  // warm
        if (st != DVG_OK) return st;
        float runs[3];
        for (int k = 0; k < 3; ++k) {
            CK(cudaEventRecord(e0, ctx->stream));
            st = run();
            if (st != DVG_OK) return st;
            CK(cudaEventRecord(e1, ctx->stream));
            CK(cudaEventSynchronize(e1));
            CK(cudaEventElapsedTime(&runs[k], e0, e1));
        }
        std::sort(runs, runs + 3);
        *ms = runs[1];
        return DVG_OK;
    };
    const uint32_t slots0 = try_slots ? 16 : 0;
    dvg_status st = DVG_OK;
    dvg_tuning best{1, 4, slots0};
    float best_ms = 0.0f, ms = 0.0f;
    auto consider = [&](dvg_tuning t) {
        if (st != DVG_OK) return;
        st = time_of(t, &ms);
        if (st == DVG_OK && ms < best_ms) {
            best = t;
            best_ms = ms;
        }
    };
    st = time_of(best, &best_ms);
    consider(dvg_tuning{0, 4, slots0});
    const uint32_t cells[3] = {2, 8, 16};
    const dvg_tuning base = best;
    for (int k = 0; k < 3; ++k) consider(dvg_tuning{base.sample_layout, cells[k], slots0});
    if (try_slots) {
        const uint32_t slots[3] = {0, 8, 32};
        const dvg_tuning b2 = best;
        for (int k = 0; k < 3; ++k) consider(dvg_tuning{b2.sample_layout, b2.boundary_cell, slots[k]});
    }
    if (try_queue) consider(dvg_tuning{best.sample_layout, best.boundary_cell, best.fragment_slots, 1, 0});
    {
        const dvg_tuning b3 = best;
        for (uint32_t occ = 1; occ <= 2; ++occ)
            consider(dvg_tuning{b3.sample_layout, b3.boundary_cell, b3.fragment_slots, b3.work_queue, occ});
    }
    *tune = best;
    if (st == DVG_OK) st = apply();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}
}  // namespace

extern "C" dvg_status dvg_scene_set_tuning(dvg_scene* scene, const dvg_tuning* tuning) {
    if (!scene || !tuning_valid(tuning)) return fail(DVG_ERR_INVALID_ARGUMENT, "invalid tuning");
    scene->tune = *tuning;
    return DVG_OK;
}
extern "C" dvg_status dvg_scene_get_tuning(const dvg_scene* scene, dvg_tuning* tuning) {
    if (!scene || !tuning) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    *tuning = scene->tune;
    return DVG_OK;
}
extern "C" dvg_status dvg_scene_autotune(dvg_context* ctx, dvg_scene* scene, const dvg_render_options* opts,
                                         const dvg_backward_options* bopts, const float* target_rgba,
                                         dvg_tuning* out) {
    if (!ctx || !scene || !target_rgba) return fail(DVG_ERR_INVALID_ARGUMENT, "null argument");
    dvg_status st = check_options(opts);
    if (st != DVG_OK) return st;
    CK(cudaSetDevice(ctx->device));
    const GradPtrs G = device_grads(scene);
    dvg_grads g{};
    g.d_shape_params = G.d_shape_params;
    g.d_shape_transform = G.d_shape_transform;
    g.d_shape_stroke_width = G.d_shape_stroke_width;
    g.d_points = G.d_points;
    g.d_thickness = G.d_thickness;
    g.d_group_transform = G.d_group_transform;
    g.d_paint_params = G.d_paint_params;
    g.d_stop_offsets = G.d_stop_offsets;
    g.d_stop_colors = G.d_stop_colors;
    g.d_filter_radius = G.d_filter_radius;
    g.d_background = G.d_background;
    st = autotune_loop(
        ctx, &scene->tune, opts->use_prefiltering == 0, []() { return DVG_OK; },
        [&]() { return dvg_fwd_bwd_l2_device(ctx, scene, opts, bopts, target_rgba, nullptr, nullptr, &g); });
    if (st != DVG_OK) return st;
    if (out) *out = scene->tune;
    return check_status(ctx);
}

extern "C" dvg_status dvg_batch_set_tuning(dvg_batch* b, const dvg_tuning* tuning) {
    if (!b || !tuning_valid(tuning)) return fail(DVG_ERR_INVALID_ARGUMENT, "invalid tuning");
    dvg_context* ctx = b->ctx;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    batch_drop_graph(b);
    b->tune = *tuning;
    // start from the device entries: the optimisation step updates some of their fields
    const size_t eb = b->host_entries.size() * sizeof(BatchEntry);
    CK(cudaMemcpyAsync(b->host_entries.data(), b->entries.ptr, eb, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    dvg_status st = batch_apply_tuning(b);
    if (st != DVG_OK) return st;
    CK(cudaMemcpyAsync(b->entries.ptr, b->host_entries.data(), eb, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return DVG_OK;
}

extern "C" dvg_status dvg_batch_autotune(dvg_batch* b, dvg_tuning* out) {
    if (!b) return fail(DVG_ERR_INVALID_ARGUMENT, "null batch");
    dvg_context* ctx = b->ctx;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    batch_drop_graph(b);
    dvg_tuning t = b->tune;
    const bool adam = b->adam;
    b->adam = false;  // time forward + loss + backward only: the parameters must not move
    dvg_status st = autotune_loop(
        ctx, &t, b->opts.use_prefiltering == 0, [&]() { return dvg_batch_set_tuning(b, &t); },
        [&]() { return batch_enqueue(b); }, true);
    b->adam = adam;
    if (st != DVG_OK) return st;
    if (out) *out = b->tune;
    return check_status(ctx);
}
