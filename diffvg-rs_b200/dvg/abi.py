"""ctypes mirror of include/dvg.h and the scene packer.

``pack_scene`` flattens a ``Scene`` into the structure-of-arrays
``dvg_scene_desc`` the C ABI takes (integer indices, one paint entry per group
fill / stroke).  ``GradBuffers`` allocates the flat ``dvg_grads`` arrays and
``unflatten_grads`` rebuilds the crate's ``SceneGrad`` shape
(src/grad.rs:113-126) from them.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from collections.abc import Sequence
from typing import Dict, List, Optional

import importlib
import itertools
import os
import subprocess

import numpy as np

from .scene import (
    BackwardOptions,
    Circle,
    Color,
    Ellipse,
    LinearGradient,
    PathGeometry,
    RadialGradient,
    Rect,
    RenderOptions,
    Scene,
)

SHAPE_CIRCLE, SHAPE_RECT, SHAPE_PATH, SHAPE_ELLIPSE = 0, 1, 2, 3
PAINT_NONE, PAINT_SOLID, PAINT_LINEAR, PAINT_RADIAL = 0, 1, 2, 3
PATH_CLOSED, PATH_DISTANCE_APPROX, PATH_HAS_THICKNESS = 1, 2, 4

_fp = C.POINTER(C.c_float)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


class SceneDesc(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("background", C.c_float * 4),
        ("background_image", _fp),
        ("filter_type", C.c_uint32), ("filter_radius", C.c_float),
        ("num_shapes", C.c_uint32),
        ("shape_kind", _u32p), ("shape_params", _fp), ("shape_transform", _fp),
        ("shape_stroke_width", _fp), ("shape_stroke_join", _u32p), ("shape_stroke_cap", _u32p),
        ("shape_miter_limit", _fp),
        ("path_ctrl_offset", _u32p), ("path_ctrl_count", _u32p),
        ("path_point_offset", _u32p), ("path_point_count", _u32p), ("path_flags", _u32p),
        ("num_control_points", _u8p), ("points", _fp), ("thickness", _fp),
        ("total_ctrl", C.c_uint32), ("total_points", C.c_uint32),
        ("num_groups", C.c_uint32),
        ("group_shape_offset", _u32p), ("group_shape_count", _u32p), ("group_shape_ids", _u32p),
        ("total_group_shapes", C.c_uint32),
        ("group_fill_rule", _u32p), ("group_shape_to_canvas", _fp), ("group_canvas_to_shape", _fp),
        ("group_fill_paint", _i32p), ("group_stroke_paint", _i32p),
        ("num_paints", C.c_uint32),
        ("paint_kind", _u32p), ("paint_params", _fp), ("paint_stop_offset", _u32p),
        ("paint_stop_count", _u32p), ("stop_offsets", _fp), ("stop_colors", _fp),
        ("total_stops", C.c_uint32),
    ]


class RenderOptionsC(C.Structure):
    _fields_ = [
        ("aa", C.c_float), ("path_tolerance", C.c_float),
        ("samples_x", C.c_uint32), ("samples_y", C.c_uint32), ("seed", C.c_uint32),
        ("jitter", C.c_uint32), ("use_prefiltering", C.c_uint32),
    ]


class BackwardOptionsC(C.Structure):
    _fields_ = [
        ("compute_translation", C.c_uint32), ("boundary_samples", C.c_uint32), ("rng", C.c_uint32),
        ("boundary_seed", C.c_uint32), ("boundary_seed_from_options", C.c_uint32),
    ]


class GradsC(C.Structure):
    _fields_ = [(n, _fp) for n in (
        "d_shape_params", "d_shape_transform", "d_shape_stroke_width", "d_points", "d_thickness",
        "d_group_transform", "d_paint_params", "d_stop_offsets", "d_stop_colors", "d_filter_radius",
        "d_background", "d_background_image", "d_translation")]


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


def render_options_c(o: RenderOptions) -> RenderOptionsC:
    return RenderOptionsC(float(o.aa), float(o.path_tolerance), int(o.samples_x), int(o.samples_y),
                          int(o.seed) & 0xFFFFFFFF, 1 if o.jitter else 0, 1 if o.use_prefiltering else 0)


def backward_options_c(b: Optional[BackwardOptions]) -> BackwardOptionsC:
    b = b or BackwardOptions()
    from_opts = 1 if b.boundary_seed is None else 0
    seed = 0 if b.boundary_seed is None else int(b.boundary_seed) & 0xFFFFFFFF
    return BackwardOptionsC(1 if b.compute_translation else 0, int(b.boundary_samples), int(b.rng), seed, from_opts)


@dataclass
class PackedScene:
    """A packed scene: the ctypes description plus the numpy arrays it points into."""

    desc: SceneDesc
    arrays: Dict[str, np.ndarray]
    # paint bookkeeping: (group index, "fill"|"stroke") -> paint index
    paint_of: Dict[tuple, int] = field(default_factory=dict)
    path_point_offset: List[int] = field(default_factory=list)
    path_point_count: List[int] = field(default_factory=list)
    stop_offset: List[int] = field(default_factory=list)
    stop_count: List[int] = field(default_factory=list)

    def ref(self):
        return C.byref(self.desc)


def _paint_record(p):
    if isinstance(p, Color):
        return PAINT_SOLID, [p.r, p.g, p.b, p.a], []
    if isinstance(p, LinearGradient):
        return PAINT_LINEAR, [p.start[0], p.start[1], p.end[0], p.end[1]], p.stops
    if isinstance(p, RadialGradient):
        return PAINT_RADIAL, [p.center[0], p.center[1], p.radius[0], p.radius[1]], p.stops
    raise TypeError(f"unsupported paint {type(p)!r}")


_PACKER = None


def _packer():
    """The native packer module (csrc/pack.cpp, built by `make -C diffvg-rs_b200 pack`
    on first use when missing) and the classes it tests against."""
    global _PACKER
    if _PACKER is None:
        try:
            from . import _dvgpack
        except ImportError:
            pkg = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
            subprocess.run(["make", "-s", "-C", pkg, "pack"], check=True)
            importlib.invalidate_caches()
            from . import _dvgpack

        def as_f32(m):
            return np.ascontiguousarray(np.asarray(m, np.float32).reshape(-1))

        _PACKER = (_dvgpack, (PathGeometry, Circle, Ellipse, Rect, Color, LinearGradient, RadialGradient, as_f32))
    return _PACKER


def pack_scene(scene: Scene) -> PackedScene:
    """Scene -> dvg_scene_desc arrays, in one native pass over the scene objects."""
    mod, types = _packer()
    raw, any_thick, paint_of = mod.pack(scene, types)

    def arr(k, dt, default=None):
        a = np.frombuffer(raw[k], dt)
        return a if a.size or default is None else np.asarray(default, dt)

    u32, f32 = np.uint32, np.float32
    n_pts = len(raw["pts"]) // 8
    g_ids = arr("g_ids", np.int64)
    arrays = dict(
        kinds=arr("kinds", u32), params=arr("params", f32), xforms=arr("xforms", f32), sw=arr("sw", f32),
        joins=arr("joins", u32), caps=arr("caps", u32), miters=arr("miters", f32), ctrl_off=arr("ctrl_off", u32),
        ctrl_cnt=arr("ctrl_cnt", u32), pt_off=arr("pt_off", u32), pt_cnt=arr("pt_cnt", u32),
        flags=arr("flags", u32), ncp=arr("ncp", np.uint8, [0]), pts=arr("pts", f32, [0.0, 0.0]),
        thick=arr("thick", f32, [0.0]),
        g_off=arr("g_off", u32), g_cnt=arr("g_cnt", u32), g_ids=(g_ids if g_ids.size else np.zeros(1, np.int64)).astype(u32),
        g_rule=arr("g_rule", u32), g_s2c=arr("g_s2c", f32), g_c2s=arr("g_c2s", f32),
        g_fill=arr("g_fill", np.int32), g_stroke=arr("g_stroke", np.int32),
        p_kind=arr("p_kind", u32, [0]), p_params=arr("p_params", f32, [0.0] * 4), p_soff=arr("p_soff", u32, [0]),
        p_scnt=arr("p_scnt", u32, [0]), s_off=arr("s_off", f32, [0.0]), s_col=arr("s_col", f32, [0.0] * 4),
    )
    counts = dict(ctrl=len(raw["ncp"]), points=n_pts, group_shapes=int(g_ids.size), paints=len(raw["p_kind"]) // 4,
                  stops=len(raw["s_off"]) // 4)
    return _describe(scene, arrays, counts, bool(any_thick), paint_of)


def pack_scene_python(scene: Scene) -> PackedScene:
    """pack_scene in plain Python (one pass collecting lists, one numpy conversion per
    array): the reference the native packer is tested against, byte for byte."""
    ns = len(scene.shapes)
    kinds: List[int] = []
    params: List[tuple] = []
    xf: List[np.ndarray] = []
    sw: List[float] = []
    joins: List[int] = []
    caps: List[int] = []
    miters: List[float] = []
    ctrl_off: List[int] = []
    ctrl_cnt: List[int] = []
    pt_off: List[int] = []
    pt_cnt: List[int] = []
    flags: List[int] = []
    ncp_l: List[int] = []
    pts_l: list = []
    th_parts: List[tuple] = []  # (point offset, thickness values) of paths that have them
    zero4 = (0.0, 0.0, 0.0, 0.0)
    for sh in scene.shapes:
        g = sh.geometry
        xf.append(sh.transform.m)
        sw.append(sh.stroke_width)
        joins.append(int(sh.stroke_join))
        caps.append(int(sh.stroke_cap))
        miters.append(sh.stroke_miter_limit)
        if isinstance(g, PathGeometry):
            p = g.path
            npt = len(p.points)
            kinds.append(SHAPE_PATH)
            params.append(zero4)
            ctrl_off.append(len(ncp_l))
            ctrl_cnt.append(len(p.num_control_points))
            pt_off.append(len(pts_l))
            pt_cnt.append(npt)
            ncp_l.extend(p.num_control_points)
            pts_l.extend(p.points)
            f = (PATH_CLOSED if p.is_closed else 0) | (PATH_DISTANCE_APPROX if p.use_distance_approx else 0)
            if p.thickness is not None:
                f |= PATH_HAS_THICKNESS
                th_parts.append((pt_off[-1], [float(x) for x in list(p.thickness)[:npt]]))
            flags.append(f)
            continue
        ctrl_off.append(0)
        ctrl_cnt.append(0)
        pt_off.append(0)
        pt_cnt.append(0)
        flags.append(0)
        if isinstance(g, Circle):
            kinds.append(SHAPE_CIRCLE)
            params.append((g.center[0], g.center[1], g.radius, 0.0))
        elif isinstance(g, Ellipse):
            kinds.append(SHAPE_ELLIPSE)
            params.append((g.center[0], g.center[1], g.radius[0], g.radius[1]))
        elif isinstance(g, Rect):
            kinds.append(SHAPE_RECT)
            params.append((g.min[0], g.min[1], g.max[0], g.max[1]))
        else:
            raise TypeError(f"unsupported geometry {type(g)!r}")
    n_ncp, n_pts = len(ncp_l), len(pts_l)
    u32 = lambda v: np.asarray(v, np.uint32).reshape(-1)  # noqa: E731
    f32 = lambda v: np.asarray(v, np.float32).reshape(-1)  # noqa: E731
    kinds, sw, joins, caps, miters = u32(kinds), f32(sw), u32(joins), u32(caps), f32(miters)
    ctrl_off, ctrl_cnt, pt_off, pt_cnt, flags = u32(ctrl_off), u32(ctrl_cnt), u32(pt_off), u32(pt_cnt), u32(flags)
    params = np.fromiter(itertools.chain.from_iterable(params), np.float32, 4 * ns).reshape(ns, 4)
    # every Mat3 holds a (3, 3) float32 array, so the rows concatenate without a copy per shape
    xforms = np.concatenate(xf).astype(np.float32, copy=False).reshape(ns, 9) if ns else np.zeros((0, 9), np.float32)
    ncp = np.asarray(ncp_l, np.int64).astype(np.uint8) if n_ncp else np.zeros(1, np.uint8)
    pts = np.fromiter(itertools.chain.from_iterable(pts_l), np.float32, 2 * n_pts) if n_pts else np.zeros(2, np.float32)
    any_thick = bool(th_parts)
    thick = np.zeros(max(n_pts, 1), np.float32)
    for o, t in th_parts:
        thick[o: o + len(t)] = t

    ng = len(scene.groups)
    g_off: List[int] = []
    g_cnt: List[int] = []
    g_ids: List[int] = []
    g_rule: List[int] = []
    s2c: List[np.ndarray] = []
    c2s: List[np.ndarray] = []
    g_fill: List[int] = []
    g_stroke: List[int] = []
    p_kind: List[int] = []
    p_params: List[List[float]] = []
    p_soff: List[int] = []
    p_scnt: List[int] = []
    s_off: List[float] = []
    s_col: List[float] = []
    paint_of = {}
    for gi, grp in enumerate(scene.groups):
        g_off.append(len(g_ids))
        g_cnt.append(len(grp.shape_indices))
        g_ids.extend(grp.shape_indices)
        g_rule.append(int(grp.fill_rule))
        s2c.append(grp.shape_to_canvas.m)
        c2s.append(grp.canvas_to_shape.m)
        for which, paint, arr in (("stroke", grp.stroke, g_stroke), ("fill", grp.fill, g_fill)):
            if paint is None:
                arr.append(-1)
                continue
            k, prm, stops = _paint_record(paint)
            arr.append(len(p_kind))
            paint_of[(gi, which)] = len(p_kind)
            p_kind.append(k)
            p_params.append(prm)
            p_soff.append(len(s_off))
            p_scnt.append(len(stops))
            for st in stops:
                s_off.append(st.offset)
                s_col += [st.color.r, st.color.g, st.color.b, st.color.a]
    g_off, g_cnt, g_rule = u32(g_off), u32(g_cnt), u32(g_rule)
    g_fill, g_stroke = np.asarray(g_fill, np.int32).reshape(-1), np.asarray(g_stroke, np.int32).reshape(-1)
    g_s2c = np.concatenate(s2c).astype(np.float32, copy=False).reshape(ng, 9) if ng else np.zeros((0, 9), np.float32)
    g_c2s = np.concatenate(c2s).astype(np.float32, copy=False).reshape(ng, 9) if ng else np.zeros((0, 9), np.float32)

    arrays = dict(
        kinds=kinds, params=params.reshape(-1), xforms=xforms.reshape(-1), sw=sw, joins=joins, caps=caps,
        miters=miters, ctrl_off=ctrl_off, ctrl_cnt=ctrl_cnt, pt_off=pt_off, pt_cnt=pt_cnt, flags=flags,
        ncp=ncp, pts=pts, thick=thick,
        g_off=g_off, g_cnt=g_cnt, g_ids=np.asarray(g_ids if g_ids else [0], np.int64).astype(np.uint32), g_rule=g_rule,
        g_s2c=g_s2c.reshape(-1), g_c2s=g_c2s.reshape(-1), g_fill=g_fill, g_stroke=g_stroke,
        p_kind=np.asarray(p_kind if p_kind else [0], np.uint32),
        p_params=np.asarray(p_params if p_params else [[0, 0, 0, 0]], np.float32).reshape(-1),
        p_soff=np.asarray(p_soff if p_soff else [0], np.uint32),
        p_scnt=np.asarray(p_scnt if p_scnt else [0], np.uint32),
        s_off=np.asarray(s_off if s_off else [0.0], np.float32),
        s_col=np.asarray(s_col if s_col else [0.0] * 4, np.float32),
    )
    counts = dict(ctrl=n_ncp, points=n_pts, group_shapes=len(g_ids), paints=len(p_kind), stops=len(s_off))
    return _describe(scene, arrays, counts, any_thick, paint_of)


def _describe(scene: Scene, arrays: Dict[str, np.ndarray], counts: Dict[str, int], any_thick: bool,
              paint_of: dict) -> PackedScene:
    """The dvg_scene_desc over packed arrays (shared by both packers)."""
    bg_img = None
    if scene.background_image is not None:
        bg_img = np.ascontiguousarray(np.asarray(scene.background_image, np.float32).reshape(-1))
        arrays["bg_img"] = bg_img

    d = SceneDesc()
    d.width, d.height = int(scene.width), int(scene.height)
    for k, v in enumerate(scene.background.to_tuple()):
        d.background[k] = float(v)
    d.background_image = _ptr(bg_img, C.c_float)
    d.filter_type = int(scene.filter.filter_type)
    d.filter_radius = float(scene.filter.radius)
    d.num_shapes = len(scene.shapes)
    d.shape_kind = _ptr(arrays["kinds"], C.c_uint32)
    d.shape_params = _ptr(arrays["params"], C.c_float)
    d.shape_transform = _ptr(arrays["xforms"], C.c_float)
    d.shape_stroke_width = _ptr(arrays["sw"], C.c_float)
    d.shape_stroke_join = _ptr(arrays["joins"], C.c_uint32)
    d.shape_stroke_cap = _ptr(arrays["caps"], C.c_uint32)
    d.shape_miter_limit = _ptr(arrays["miters"], C.c_float)
    d.path_ctrl_offset = _ptr(arrays["ctrl_off"], C.c_uint32)
    d.path_ctrl_count = _ptr(arrays["ctrl_cnt"], C.c_uint32)
    d.path_point_offset = _ptr(arrays["pt_off"], C.c_uint32)
    d.path_point_count = _ptr(arrays["pt_cnt"], C.c_uint32)
    d.path_flags = _ptr(arrays["flags"], C.c_uint32)
    d.num_control_points = _ptr(arrays["ncp"], C.c_uint8)
    d.points = _ptr(arrays["pts"], C.c_float)
    d.thickness = _ptr(arrays["thick"], C.c_float) if any_thick else C.cast(None, _fp)
    d.total_ctrl = counts['ctrl']
    d.total_points = counts['points']
    d.num_groups = len(scene.groups)
    d.group_shape_offset = _ptr(arrays["g_off"], C.c_uint32)
    d.group_shape_count = _ptr(arrays["g_cnt"], C.c_uint32)
    d.group_shape_ids = _ptr(arrays["g_ids"], C.c_uint32)
    d.total_group_shapes = counts['group_shapes']
    d.group_fill_rule = _ptr(arrays["g_rule"], C.c_uint32)
    d.group_shape_to_canvas = _ptr(arrays["g_s2c"], C.c_float)
    d.group_canvas_to_shape = _ptr(arrays["g_c2s"], C.c_float)
    d.group_fill_paint = _ptr(arrays["g_fill"], C.c_int32)
    d.group_stroke_paint = _ptr(arrays["g_stroke"], C.c_int32)
    d.num_paints = counts['paints']
    d.paint_kind = _ptr(arrays["p_kind"], C.c_uint32)
    d.paint_params = _ptr(arrays["p_params"], C.c_float)
    d.paint_stop_offset = _ptr(arrays["p_soff"], C.c_uint32)
    d.paint_stop_count = _ptr(arrays["p_scnt"], C.c_uint32)
    d.stop_offsets = _ptr(arrays["s_off"], C.c_float)
    d.stop_colors = _ptr(arrays["s_col"], C.c_float)
    d.total_stops = counts['stops']
    soff = arrays["p_soff"][: counts["paints"]].tolist()
    scnt = arrays["p_scnt"][: counts["paints"]].tolist()
    return PackedScene(d, arrays, paint_of, arrays["pt_off"].tolist(), arrays["pt_cnt"].tolist(), soff, scnt)


class GradBuffers:
    """Host arrays behind a dvg_grads struct, sized from a packed scene."""

    NAMES = ("d_shape_params", "d_shape_transform", "d_shape_stroke_width", "d_points", "d_thickness",
             "d_group_transform", "d_paint_params", "d_stop_offsets", "d_stop_colors", "d_filter_radius",
             "d_background", "d_background_image", "d_translation")

    def __init__(self, packed: PackedScene, background_image: bool = False, translation: bool = False):
        d = packed.desc
        npix = int(d.width) * int(d.height)
        sizes = dict(
            d_shape_params=4 * d.num_shapes, d_shape_transform=9 * d.num_shapes,
            d_shape_stroke_width=d.num_shapes, d_points=2 * d.total_points, d_thickness=d.total_points,
            d_group_transform=9 * d.num_groups, d_paint_params=4 * d.num_paints, d_stop_offsets=d.total_stops,
            d_stop_colors=4 * d.total_stops, d_filter_radius=1, d_background=4,
            d_background_image=4 * npix if background_image else 0, d_translation=2 * npix if translation else 0,
        )
        self.arrays: Dict[str, Optional[np.ndarray]] = {}
        self.c = GradsC()
        for n in self.NAMES:
            sz = sizes[n]
            if n in ("d_background_image", "d_translation") and sz == 0:
                self.arrays[n] = None
                setattr(self.c, n, C.cast(None, _fp))
                continue
            a = np.zeros(max(int(sz), 1), np.float32)
            self.arrays[n] = a
            setattr(self.c, n, _ptr(a, C.c_float))

    def __getitem__(self, k: str) -> Optional[np.ndarray]:
        return self.arrays[k]

    def flat(self) -> np.ndarray:
        """All gradient values concatenated (for norms / relative-error checks)."""
        parts = [a for a in self.arrays.values() if a is not None]
        return np.concatenate(parts) if parts else np.zeros(0, np.float32)


@dataclass
class DShape:
    geometry: dict
    transform: np.ndarray
    stroke_width: float


@dataclass
class DShapeGroup:
    shape_to_canvas: np.ndarray
    fill: Optional[dict]
    stroke: Optional[dict]


@dataclass
class SceneGrad:
    """src/grad.rs:113-126, with numpy leaves."""

    shapes: List[DShape]
    shape_groups: List[DShapeGroup]
    filter_radius: float
    background: np.ndarray
    background_image: Optional[np.ndarray]
    translation: Optional[np.ndarray]
    buffers: GradBuffers

    def to_diffvg_layout(self, scene: Scene) -> "DiffvgSceneGrad":
        return to_diffvg_layout(self, scene)


@dataclass
class DiffvgShapeGrad:
    """src/grad.rs (DiffvgShapeGrad): geometry gradient with path metadata."""

    geometry: dict
    transform: np.ndarray
    stroke_width: float


@dataclass
class DiffvgSceneGrad:
    """src/grad.rs:451-466: the diffvg-compatible gradient layout."""

    shapes: List[DiffvgShapeGrad]
    shape_groups: List[DShapeGroup]
    filter_radius: float
    background: np.ndarray
    background_image: Optional[np.ndarray]
    translation: Optional[np.ndarray]


def to_diffvg_layout(grad: "SceneGrad", scene: Scene) -> DiffvgSceneGrad:
    """SceneGrad::to_diffvg_layout (src/grad.rs:474-553): path gradients carry the
    path's control-point counts, closure and distance-approximation flag, and
    per-point buffers take the source path's lengths (zero-padded or truncated)."""
    shapes = []
    for idx, ds in enumerate(grad.shapes):
        g = dict(ds.geometry)
        src = scene.shapes[idx].geometry if idx < len(scene.shapes) else None
        if g["kind"] == "path":
            path = getattr(src, "path", None)
            if path is not None:
                pts = np.zeros((len(path.points), 2), np.float32)
                n = min(len(path.points), len(g["points"]))
                pts[:n] = g["points"][:n]
                th = g.get("thickness")
                if path.thickness is not None:
                    out_th = np.zeros(len(path.thickness), np.float32)
                    if th is not None:
                        m = min(len(out_th), len(th))
                        out_th[:m] = th[:m]
                    th = out_th
                g = dict(kind="path", num_control_points=list(path.num_control_points), points=pts, thickness=th,
                         is_closed=bool(path.is_closed), use_distance_approx=bool(path.use_distance_approx))
            else:
                g = dict(kind="path", num_control_points=[], points=g["points"], thickness=g.get("thickness"),
                         is_closed=False, use_distance_approx=False)
        shapes.append(DiffvgShapeGrad(g, ds.transform, ds.stroke_width))
    groups = [DShapeGroup(gg.shape_to_canvas, gg.fill, gg.stroke) for gg in grad.shape_groups]
    return DiffvgSceneGrad(shapes, groups, grad.filter_radius, grad.background, grad.background_image,
                           grad.translation)


class LazyList(Sequence):
    """Read-only list whose items are built on first access.  A scene of thousands of
    shapes has thousands of small gradient records; building them all after every
    backward pass costs more host time than the pass's own host work, and an optimiser
    that reads the flat buffers never needs them."""

    __slots__ = ("_make", "_items")

    def __init__(self, n: int, make):
        self._make = make
        self._items = [None] * n

    def __len__(self) -> int:
        return len(self._items)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(len(self._items)))]
        it = self._items[i]  # IndexError for out-of-range indices, as a list
        if it is None:
            i = int(i) + len(self._items) if i < 0 else int(i)
            it = self._items[i] = self._make(i)
        return it

    def __iter__(self):
        return (self[i] for i in range(len(self._items)))

    def __repr__(self) -> str:
        return repr(list(self))


def _paint_grad(kind: int, buf: GradBuffers, pi: int, soff: int, scnt: int) -> dict:
    pp = buf["d_paint_params"][4 * pi: 4 * pi + 4].copy()
    stops = [dict(offset=float(buf["d_stop_offsets"][soff + k]), color=buf["d_stop_colors"][4 * (soff + k): 4 * (soff + k) + 4].copy())
             for k in range(scnt)]
    if kind == PAINT_SOLID:
        return dict(kind="solid", color=pp)
    if kind == PAINT_LINEAR:
        return dict(kind="linear", start=pp[:2], end=pp[2:], stops=stops)
    return dict(kind="radial", center=pp[:2], radius=pp[2:], stops=stops)


def unflatten_grads(scene: Scene, packed: PackedScene, buf: GradBuffers) -> SceneGrad:
    """Flat gradient buffers -> SceneGrad (src/grad.rs:113-126).  The per-shape and
    per-group records are built when first read, from the packed arrays alone (editing
    `scene` afterwards does not change them)."""
    kinds, flags = packed.arrays["kinds"], packed.arrays["flags"]
    p_kind = packed.arrays["p_kind"]
    g_fill, g_stroke = packed.arrays["g_fill"], packed.arrays["g_stroke"]

    def shape(i: int) -> DShape:
        sp = buf["d_shape_params"][4 * i: 4 * i + 4]
        k = int(kinds[i])
        if k == SHAPE_CIRCLE:
            geo = dict(kind="circle", center=sp[:2].copy(), radius=float(sp[2]))
        elif k == SHAPE_ELLIPSE:
            geo = dict(kind="ellipse", center=sp[:2].copy(), radius=sp[2:].copy())
        elif k == SHAPE_RECT:
            geo = dict(kind="rect", min=sp[:2].copy(), max=sp[2:].copy())
        else:
            o, n = packed.path_point_offset[i], packed.path_point_count[i]
            pts = buf["d_points"][2 * o: 2 * (o + n)].reshape(-1, 2).copy()
            th = buf["d_thickness"][o: o + n].copy() if int(flags[i]) & PATH_HAS_THICKNESS else None
            geo = dict(kind="path", points=pts, thickness=th)
        return DShape(geo, buf["d_shape_transform"][9 * i: 9 * i + 9].reshape(3, 3).copy(),
                      float(buf["d_shape_stroke_width"][i]))

    def paint(pi: int) -> Optional[dict]:
        if pi < 0:
            return None
        return _paint_grad(int(p_kind[pi]), buf, pi, packed.stop_offset[pi], packed.stop_count[pi])

    def group(gi: int) -> DShapeGroup:
        return DShapeGroup(buf["d_group_transform"][9 * gi: 9 * gi + 9].reshape(3, 3).copy(),
                           paint(int(g_fill[gi])), paint(int(g_stroke[gi])))

    bgi = buf["d_background_image"]
    tr = buf["d_translation"]
    return SceneGrad(LazyList(len(scene.shapes), shape), LazyList(len(scene.groups), group),
                     float(buf["d_filter_radius"][0]), buf["d_background"].copy(),
                     None if bgi is None else bgi.copy(), None if tr is None else tr.copy(), buf)


def scene_with_params(scene: Scene, packed: PackedScene, points: np.ndarray,
                      paint_params: Optional[np.ndarray] = None) -> Scene:
    """A copy of `scene` whose path points (flat [total_points, 2], as packed) and,
    if given, paint parameters ([num_paints, 4], as packed) are replaced — e.g. with
    the values a batch's on-device optimisation step reached."""
    import copy

    out = copy.deepcopy(scene)
    pts = np.asarray(points, np.float32).reshape(-1, 2)
    for si, shp in enumerate(out.shapes):
        path = getattr(shp.geometry, "path", None)
        if path is None:
            continue
        o = packed.path_point_offset[si]
        path.points = [(float(x), float(y)) for x, y in pts[o:o + len(path.points)]]
    if paint_params is not None:
        pp = np.asarray(paint_params, np.float32).reshape(-1, 4)
        for (gi, which), pi in packed.paint_of.items():
            paint = getattr(out.groups[gi], which)
            v = [float(x) for x in pp[pi]]
            if isinstance(paint, Color):
                paint.r, paint.g, paint.b, paint.a = v
            elif isinstance(paint, LinearGradient):
                paint.start, paint.end = (v[0], v[1]), (v[2], v[3])
            elif isinstance(paint, RadialGradient):
                paint.center, paint.radius = (v[0], v[1]), (v[2], v[3])
    return out
