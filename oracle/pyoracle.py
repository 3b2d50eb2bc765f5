"""ctypes binding of the CPU oracle (test infrastructure only).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference arm.  It builds oracle/_build/liboracle.so with the committed
Makefile when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.dirname(_HERE)
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
sys.path.insert(0, os.path.join(_REPO, "diffvg-rs_b200"))

from dvg.abi import (  # noqa: E402
    BackwardOptionsC,
    GradBuffers,
    GradsC,
    RenderOptionsC,
    SceneDesc,
    backward_options_c,
    pack_scene,
    render_options_c,
    unflatten_grads,
)
from dvg.scene import BackwardOptions, RenderOptions, Scene  # noqa: E402

_lib: Optional[C.CDLL] = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "oracle.cpp")
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
            build()
        L = C.CDLL(_LIB_PATH)
        D = C.POINTER(SceneDesc)
        R = C.POINTER(RenderOptionsC)
        B = C.POINTER(BackwardOptionsC)
        fp = C.POINTER(C.c_float)
        L.oracle_render.argtypes = [D, R, fp]
        L.oracle_render_window.argtypes = [D, R, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, fp]
        L.oracle_render_differentiated.argtypes = [D, R, fp]
        L.oracle_render_sdf.argtypes = [D, R, fp]
        L.oracle_lbvh_build.argtypes = [fp, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_int32), fp]
        L.oracle_eval_positions.argtypes = [D, fp, C.c_uint64, fp]
        L.oracle_sdf_backward.argtypes = [D, R, B, fp, C.POINTER(GradsC)]
        L.oracle_positions_backward.argtypes = [D, B, fp, C.c_uint64, fp, C.POINTER(GradsC)]
        L.oracle_sample_premultiplied.argtypes = [D, R, C.c_float, C.c_float, fp]
        L.oracle_render_backward.argtypes = [D, R, B, fp, C.POINTER(GradsC)]
        L.oracle_render_backward_ex.argtypes = [D, R, B, fp, C.POINTER(GradsC), C.c_int, C.c_int,
                                                C.c_ulonglong, C.c_ulonglong]
        L.oracle_weight_image.argtypes = [D, R, fp]
        L.oracle_boundary_integral.argtypes = [D, R, fp, C.c_uint32, C.c_float, C.c_int, C.POINTER(GradsC)]
        L.oracle_compute_distance.argtypes = [D, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_int, fp]
        L.oracle_within_distance.argtypes = [D, C.c_uint32, C.c_float, C.c_float, C.c_int]
        L.oracle_is_inside.argtypes = [D, C.c_uint32, C.c_float, C.c_float, C.c_int]
        L.oracle_flatten.argtypes = [D, C.c_uint32, C.c_float, fp, C.c_int]
        L.oracle_pcg32_floats.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_int, fp]
        L.oracle_philox_floats.argtypes = [C.c_ulonglong, C.c_uint, fp]
        L.oracle_path_bvh.argtypes = [D, C.c_uint32, fp, C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]
        L.oracle_fwd_bwd_sample.argtypes = [D, R, B, fp, C.c_ulonglong, C.c_int, C.POINTER(C.c_double)]
        L.oracle_fwd_bwd_sample.restype = C.c_ulonglong
        _lib = L
    return _lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def render(scene: Scene, options: RenderOptions) -> np.ndarray:
    ps = pack_scene(scene)
    out = np.zeros(int(scene.width) * int(scene.height) * 4, np.float32)
    o = render_options_c(options)
    lib().oracle_render(ps.ref(), C.byref(o), _fp(out))
    return out.reshape(int(scene.height), int(scene.width), 4)


def render_window(scene: Scene, options: RenderOptions, x0: int, y0: int, x1: int, y1: int,
                  threads: int = 0) -> np.ndarray:
    """Pixels [x0,x1) x [y0,y1) of render() ([y1-y0, x1-x0, 4], bit-identical), the
    per-sample colours on `threads` host threads (0: every core)."""
    ps = pack_scene(scene)
    x1, y1 = min(x1, int(scene.width)), min(y1, int(scene.height))
    out = np.zeros(max(x1 - x0, 0) * max(y1 - y0, 0) * 4, np.float32)
    o = render_options_c(options)
    lib().oracle_render_window(ps.ref(), C.byref(o), x0, y0, x1, y1, threads or (os.cpu_count() or 1), _fp(out))
    return out.reshape(max(y1 - y0, 0), max(x1 - x0, 0), 4)


def render_differentiated(scene: Scene, options: RenderOptions) -> np.ndarray:
    """The image render_backward differentiates: per pixel, the filter-weighted
    average of per-sample un-premultiplied colours (equal to render() wherever
    every sample of a pixel is opaque)."""
    ps = pack_scene(scene)
    out = np.zeros(int(scene.width) * int(scene.height) * 4, np.float32)
    o = render_options_c(options)
    lib().oracle_render_differentiated(ps.ref(), C.byref(o), _fp(out))
    return out.reshape(int(scene.height), int(scene.width), 4)


def sample_premultiplied(scene: Scene, px: float, py: float) -> np.ndarray:
    ps = pack_scene(scene)
    out = np.zeros(4, np.float32)
    o = render_options_c(RenderOptions())
    lib().oracle_sample_premultiplied(ps.ref(), C.byref(o), px, py, _fp(out))
    return out


def weight_image(scene: Scene, options: RenderOptions) -> np.ndarray:
    ps = pack_scene(scene)
    out = np.zeros(int(scene.width) * int(scene.height), np.float32)
    o = render_options_c(options)
    lib().oracle_weight_image(ps.ref(), C.byref(o), _fp(out))
    return out.reshape(int(scene.height), int(scene.width))


def render_backward(scene: Scene, options: RenderOptions, bopts: Optional[BackwardOptions] = None,
                    d_render: Optional[np.ndarray] = None, passes: int = 3, threads: int = 1,
                    sample_begin: int = 0, sample_end: int = 0):
    """The crate's CPU render_backward; returns (SceneGrad, GradBuffers)."""
    bopts = bopts or BackwardOptions()
    ps = pack_scene(scene)
    has_bg = d_render is not None and scene.background_image is not None
    buf = GradBuffers(ps, background_image=has_bg, translation=bopts.compute_translation)
    o = render_options_c(options)
    b = backward_options_c(bopts)
    dr = None
    if d_render is not None:
        dr = np.ascontiguousarray(np.asarray(d_render, np.float32).reshape(-1))
    lib().oracle_render_backward_ex(ps.ref(), C.byref(o), C.byref(b),
                                    _fp(dr) if dr is not None else C.cast(None, C.POINTER(C.c_float)),
                                    C.byref(buf.c), passes, threads, sample_begin, sample_end)
    return unflatten_grads(scene, ps, buf), buf


def boundary_integral(scene: Scene, options: RenderOptions, d_render: np.ndarray, m: int,
                      offset: float = 1.0e-4, threads: int = 0):
    """Expectation over boundary seeds of the crate's boundary gradients (midpoint rule
    with m steps of every shape's boundary parameter; see oracle_boundary_integral).
    offset: the colour-sampling offset in normalised canvas units.  Returns
    (SceneGrad, GradBuffers) as render_backward."""
    ps = pack_scene(scene)
    buf = GradBuffers(ps, background_image=False, translation=False)
    o = render_options_c(options)
    dr = np.ascontiguousarray(np.asarray(d_render, np.float32).reshape(-1))
    lib().oracle_boundary_integral(ps.ref(), C.byref(o), _fp(dr), m, offset, threads or (os.cpu_count() or 1),
                                   C.byref(buf.c))
    return unflatten_grads(scene, ps, buf), buf


def render_sdf(scene: Scene, options: RenderOptions) -> np.ndarray:
    """Renderer::render_sdf: per-pixel mean signed distance, [height, width]."""
    ps = pack_scene(scene)
    out = np.zeros(int(scene.width) * int(scene.height), np.float32)
    o = render_options_c(options)
    lib().oracle_render_sdf(ps.ref(), C.byref(o), _fp(out))
    return out.reshape(int(scene.height), int(scene.width))


def eval_positions(scene: Scene, positions) -> np.ndarray:
    """Renderer::eval_positions: signed distance at each canvas point ([n, 2] -> [n])."""
    ps = pack_scene(scene)
    pos = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1))
    out = np.zeros(pos.size // 2, np.float32)
    lib().oracle_eval_positions(ps.ref(), _fp(pos), out.size, _fp(out))
    return out


def sdf_backward(scene: Scene, options: RenderOptions, bopts: Optional[BackwardOptions], d_sdf: np.ndarray):
    """The d_sdf_image part of the crate's render_backward; returns (SceneGrad, GradBuffers)."""
    bopts = bopts or BackwardOptions()
    ps = pack_scene(scene)
    buf = GradBuffers(ps, background_image=False, translation=bopts.compute_translation)
    o = render_options_c(options)
    b = backward_options_c(bopts)
    d = np.ascontiguousarray(np.asarray(d_sdf, np.float32).reshape(-1))
    lib().oracle_sdf_backward(ps.ref(), C.byref(o), C.byref(b), _fp(d), C.byref(buf.c))
    return unflatten_grads(scene, ps, buf), buf


def eval_positions_backward(scene: Scene, positions, bopts: Optional[BackwardOptions], d_values):
    """render_backward_positions; returns (SceneGrad, GradBuffers)."""
    bopts = bopts or BackwardOptions()
    ps = pack_scene(scene)
    buf = GradBuffers(ps, background_image=False, translation=bopts.compute_translation)
    b = backward_options_c(bopts)
    pos = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1))
    d = np.ascontiguousarray(np.asarray(d_values, np.float32).reshape(-1))
    lib().oracle_positions_backward(ps.ref(), C.byref(b), _fp(pos), d.size, _fp(d), C.byref(buf.c))
    return unflatten_grads(scene, ps, buf), buf


def lbvh_build(boxes: np.ndarray):
    """CPU twin of dvg_lbvh_build: (sorted keys [n], children [n-1, 2], bounds [2n-1, 4])."""
    b = np.ascontiguousarray(np.asarray(boxes, np.float32).reshape(-1, 4))
    n = b.shape[0]
    keys = np.zeros(n, np.uint64)
    ch = np.zeros((max(n - 1, 0), 2), np.int32)
    bounds = np.zeros((max(2 * n - 1, 0), 4), np.float32)
    lib().oracle_lbvh_build(_fp(b), n, keys.ctypes.data_as(C.POINTER(C.c_uint64)),
                            ch.ctypes.data_as(C.POINTER(C.c_int32)), _fp(bounds))
    return keys, ch, bounds


def compute_distance(scene: Scene, group: int, pt, max_radius: float = float("inf"), use_bvh: bool = False):
    ps = pack_scene(scene)
    out = np.zeros(4, np.float32)
    ok = lib().oracle_compute_distance(ps.ref(), group, pt[0], pt[1], max_radius, 1 if use_bvh else 0, _fp(out))
    if not ok:
        return None
    return dict(shape_index=int(out[0]), point=(float(out[1]), float(out[2])), distance=float(out[3]))


def within_distance(scene: Scene, group: int, pt, use_bvh: bool = False) -> bool:
    ps = pack_scene(scene)
    return bool(lib().oracle_within_distance(ps.ref(), group, pt[0], pt[1], 1 if use_bvh else 0))


def is_inside(scene: Scene, group: int, pt, use_bvh: bool = False) -> bool:
    ps = pack_scene(scene)
    return bool(lib().oracle_is_inside(ps.ref(), group, pt[0], pt[1], 1 if use_bvh else 0))


def flatten(scene: Scene, shape: int, tolerance: float) -> np.ndarray:
    ps = pack_scene(scene)
    cap = 1 << 16
    out = np.zeros(cap * 4, np.float32)
    n = lib().oracle_flatten(ps.ref(), shape, tolerance, _fp(out), cap)
    return out[: 4 * min(n, cap)].reshape(-1, 4)


def pcg32_floats(idx: int, seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    lib().oracle_pcg32_floats(idx, seed, n, _fp(out))
    return out


def philox_floats(idx: int, seed: int) -> np.ndarray:
    out = np.zeros(2, np.float32)
    lib().oracle_philox_floats(idx, seed, _fp(out))
    return out


def path_bvh(scene: Scene, shape: int):
    ps = pack_scene(scene)
    nodes = np.zeros(8 * 4096, np.float32)
    idx = np.zeros(4096, np.int32)
    ni = C.c_int(0)
    n = lib().oracle_path_bvh(ps.ref(), shape, _fp(nodes), 4096, idx.ctypes.data_as(C.POINTER(C.c_int)), 4096,
                              C.byref(ni))
    return nodes[: 8 * n].reshape(-1, 8), idx[: ni.value]


WORK_KINDS = ("fill_line", "fill_quad", "fill_cubic", "stroke_line", "stroke_quad", "stroke_cubic",
              "fill_circle", "fill_ellipse", "fill_rect", "stroke_circle", "stroke_ellipse", "stroke_rect")
_ops_lib: Optional[C.CDLL] = None


def count_work(scene: Scene, options: RenderOptions, threads: int = 0):
    """Forward-pass work for the compute roofline: {kind: (tests, flops)} from the
    counting build of the oracle (liboracle_ops.so; see oracle_count_work)."""
    global _ops_lib
    if _ops_lib is None:
        build()
        _ops_lib = C.CDLL(os.path.join(_HERE, "_build", "liboracle_ops.so"))
        _ops_lib.oracle_count_work.argtypes = [C.POINTER(SceneDesc), C.POINTER(RenderOptionsC), C.c_int,
                                               C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
    ps = pack_scene(scene)
    o = render_options_c(options)
    counts = (C.c_ulonglong * 12)()
    flops = (C.c_ulonglong * 12)()
    rc = _ops_lib.oracle_count_work(ps.ref(), C.byref(o), threads or (os.cpu_count() or 1), counts, flops)
    if rc != 0:
        raise RuntimeError("liboracle_ops.so was not built with operation counting")
    return {k: (int(counts[i]), int(flops[i])) for i, k in enumerate(WORK_KINDS)}


def fwd_bwd_sample(scene: Scene, options: RenderOptions, bopts: Optional[BackwardOptions], d_render: np.ndarray,
                   count: int, threads: int):
    """Bounded-sample CPU forward + backward (the CPU baseline workload).

    Returns (samples done, set-up seconds, sample-loop seconds)."""
    ps = pack_scene(scene)
    o = render_options_c(options)
    b = backward_options_c(bopts or BackwardOptions())
    dr = np.ascontiguousarray(np.asarray(d_render, np.float32).reshape(-1))
    t = (C.c_double * 2)()
    n = int(lib().oracle_fwd_bwd_sample(ps.ref(), C.byref(o), C.byref(b), _fp(dr), count, threads, t))
    return n, float(t[0]), float(t[1])
