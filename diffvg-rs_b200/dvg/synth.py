"""Seeded synthetic scenes with the shapes, sizes and value distributions of the
benchmark workloads (no dataset is involved; every scene comes from a numpy
PCG64 generator and a fixed seed).

* ``plain_scene``      256x256, 2x2 spp, box r=0.5, white background, 16 closed
                       cubic paths of 4-8 segments, points U[0,256), solid RGBA
                       fill (alpha U[0.3,1]), non-zero rule.
* ``mixed_scene``      512x512, 4x4 spp, Gaussian r=1: 128 filled closed cubic
                       paths (4-16 segments), 64 stroked open polylines /
                       quadratic paths (width U[1,6]), 32 circles (r U[4,64]),
                       32 ellipses; half even-odd; linear / radial gradient fills
                       with 2-4 sorted stops; per-group rotation U[0,2pi) and
                       scale U[0.5,2].
* ``adjoint_scene``    128x128, 4x4 spp, 4 filled cubic + 4 stroked quadratic
                       paths (width U[2,4]), solid colours.
* ``batched_scenes``   side in {128,256,512}, log-uniform shape count 4-1024 of
                       the plain mix, 4x4 spp.
* ``primitives_scene`` 64x64: one of each primitive (circle, stroked ellipse,
                       rotated rect, mixed-order closed path, open path with
                       per-point thickness), linear / radial / solid paints,
                       even-odd group with a shape-to-canvas transform.
* ``large_scene``      1024x1024, 4x4 spp, 4096 closed cubic paths of 16
                       segments, 25% stroked (width U[0.5,8]), radial 3-stop
                       fills, group and shape transforms.
* ``styled_stroke_scene`` stroked open and closed paths (lines, quadratics,
                       cubics; some with per-point thickness) with every join
                       (miter with limits U[1,6], bevel, round) and cap (butt,
                       square, round), translucent solid strokes, a few filled.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .scene import (Circle, Color, Ellipse, Filter, FilterType, FillRule, GradientStop, LinearGradient, Mat3,
                    Path, PathGeometry, RadialGradient, Rect, RenderOptions, Scene, Shape, ShapeGroup, StrokeCap,
                    StrokeJoin)


def _closed_cubic(rng: np.random.Generator, nseg: int, lo, hi) -> Path:
    pts = rng.uniform(lo, hi, size=(3 * nseg, 2)).astype(np.float32)
    return Path([2] * nseg, [tuple(map(float, p)) for p in pts], None, True, False)


def _solid(rng: np.random.Generator) -> Color:
    r, g, b = rng.uniform(0.0, 1.0, 3)
    a = rng.uniform(0.3, 1.0)
    return Color(float(np.float32(r)), float(np.float32(g)), float(np.float32(b)), float(np.float32(a)))


def _stops(rng: np.random.Generator, n: int) -> List[GradientStop]:
    offs = np.sort(rng.uniform(0.0, 1.0, n)).astype(np.float32)
    return [GradientStop(float(o), _solid(rng)) for o in offs]


def plain_scene(seed: int = 0, width: int = 256, height: int = 256, num_paths: int = 16,
                extent: float = 1.0) -> Scene:
    """``extent`` < 1 confines each path's control points to a random square of that
    fraction of the canvas (1.0: points uniform over the whole canvas)."""
    rng = np.random.default_rng(seed)
    sc = Scene(width, height)
    sc.background = Color(1.0, 1.0, 1.0, 1.0)
    sc.filter = Filter(FilterType.BOX, 0.5)
    side = float(max(width, height))
    for i in range(num_paths):
        nseg = int(rng.integers(4, 9))
        if extent >= 1.0:
            path = _closed_cubic(rng, nseg, 0.0, side)
        else:
            size = extent * side
            ox, oy = rng.uniform(0.0, side - size, 2)
            path = _closed_cubic(rng, nseg, 0.0, size)
            path.points = [(float(np.float32(x + ox)), float(np.float32(y + oy))) for x, y in path.points]
        sc.shapes.append(Shape(PathGeometry(path)))
        sc.groups.append(ShapeGroup([i], _solid(rng), None))
    return sc


def plain_options() -> RenderOptions:
    return RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=True, use_prefiltering=False)


def _group_xform(rng: np.random.Generator, width: int, height: int) -> Mat3:
    cx, cy = rng.uniform(0.0, width), rng.uniform(0.0, height)
    theta = rng.uniform(0.0, 2.0 * math.pi)
    s = rng.uniform(0.5, 2.0)
    return Mat3.translate(float(cx), float(cy)).mul(Mat3.rotate(float(theta))).mul(Mat3.scale(float(s), float(s)))


def _gradient(rng: np.random.Generator, center: Tuple[float, float], extent: float):
    n = int(rng.integers(2, 5))
    if rng.uniform() < 0.5:
        a = (center[0] - extent * float(rng.uniform(0.2, 1.0)), center[1] - extent * float(rng.uniform(0.2, 1.0)))
        b = (center[0] + extent * float(rng.uniform(0.2, 1.0)), center[1] + extent * float(rng.uniform(0.2, 1.0)))
        return LinearGradient(a, b, _stops(rng, n))
    r = extent * float(rng.uniform(0.5, 1.5))
    return RadialGradient(center, (r, r * float(rng.uniform(0.5, 1.5))), _stops(rng, n))


def mixed_scene(seed: int = 0, width: int = 512, height: int = 512, scale: float = 1.0,
                size_scale: float = 1.0) -> Scene:
    """``scale`` multiplies the shape counts and ``size_scale`` the shape sizes
    (both 1.0 for the benchmark workload; smaller for oracle-sized test cases)."""
    rng = np.random.default_rng(seed)
    sc = Scene(width, height)
    sc.background = Color(1.0, 1.0, 1.0, 1.0)
    sc.filter = Filter(FilterType.GAUSSIAN, 1.0)
    n = [max(1, int(round(c * scale))) for c in (128, 64, 32, 32)]
    kinds = ["cubic"] * n[0] + ["stroke"] * n[1] + ["circle"] * n[2] + ["ellipse"] * n[3]
    order = rng.permutation(len(kinds))
    for k in order:
        kind = kinds[k]
        xf = _group_xform(rng, width, height)
        center = xf.transform_point((0.0, 0.0))
        if kind == "cubic":
            r = float(rng.uniform(16.0, 64.0)) * size_scale
            geom = PathGeometry(_closed_cubic(rng, int(rng.integers(4, 17)), -r, r))
            ext = r
            stroke_w = 0.0
        elif kind == "stroke":
            r = float(rng.uniform(16.0, 64.0)) * size_scale
            nseg = int(rng.integers(2, 9))
            quad = rng.uniform() < 0.5
            ncp = [1 if quad else 0] * nseg
            npts = nseg * (2 if quad else 1) + 1
            pts = rng.uniform(-r, r, size=(npts, 2)).astype(np.float32)
            geom = PathGeometry(Path(ncp, [tuple(map(float, p)) for p in pts], None, False, False))
            ext = r
            stroke_w = float(np.float32(rng.uniform(1.0, 6.0)))
        elif kind == "circle":
            rad = float(np.float32(rng.uniform(4.0, 64.0) * size_scale))
            geom = Circle((0.0, 0.0), rad)
            ext = rad
            stroke_w = 0.0
        else:
            rx, ry = (float(np.float32(v * size_scale)) for v in rng.uniform(4.0, 64.0, 2))
            geom = Ellipse((0.0, 0.0), (rx, ry))
            ext = max(rx, ry)
            stroke_w = 0.0
        shape = Shape(geom)
        shape.stroke_width = stroke_w
        sid = len(sc.shapes)
        sc.shapes.append(shape)
        if kind == "stroke":
            grp = ShapeGroup([sid], None, _solid(rng))
        else:
            grp = ShapeGroup([sid], _gradient(rng, center, 2.0 * ext), None)
            grp.fill_rule = FillRule.EVEN_ODD if rng.uniform() < 0.5 else FillRule.NON_ZERO
        grp.set_shape_to_canvas(xf)
        sc.groups.append(grp)
    return sc


def mixed_options() -> RenderOptions:
    return RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=True, use_prefiltering=False)


def adjoint_scene(seed: int = 0, width: int = 128, height: int = 128) -> Scene:
    rng = np.random.default_rng(seed)
    sc = Scene(width, height)
    sc.background = Color(1.0, 1.0, 1.0, 1.0)
    sc.filter = Filter(FilterType.BOX, 0.5)
    for i in range(4):
        sc.shapes.append(Shape(PathGeometry(_closed_cubic(rng, int(rng.integers(4, 8)), 8.0, float(width - 8)))))
        sc.groups.append(ShapeGroup([len(sc.shapes) - 1], _solid(rng), None))
    for i in range(4):
        nseg = int(rng.integers(2, 5))
        pts = rng.uniform(8.0, width - 8.0, size=(2 * nseg + 1, 2)).astype(np.float32)
        shape = Shape(PathGeometry(Path([1] * nseg, [tuple(map(float, p)) for p in pts], None, False, False)))
        shape.stroke_width = float(np.float32(rng.uniform(2.0, 4.0)))
        sc.shapes.append(shape)
        sc.groups.append(ShapeGroup([len(sc.shapes) - 1], None, _solid(rng)))
    return sc


def adjoint_options() -> RenderOptions:
    return RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=True, use_prefiltering=False)


def batched_scenes(seed: int = 0, count: int = 64) -> List[Scene]:
    """Uneven batch: side in {128,256,512}, log-uniform 4-1024 paths of the plain mix.
    Paths shrink as sqrt(16/n) of the canvas above 16 paths, which keeps the depth
    complexity of the 16-path plain scene instead of stacking hundreds of
    full-canvas paths on every pixel."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        side = int(rng.choice([128, 256, 512]))
        n = int(round(math.exp(rng.uniform(math.log(4), math.log(1024)))))
        extent = min(1.0, math.sqrt(16.0 / n))
        out.append(plain_scene(int(rng.integers(0, 2 ** 31)), side, side, n, extent))
    return out


def small_scenes(seed: int = 0, count: int = 256) -> List[Scene]:
    """Many small scenes (64x64, 4-16 paths of the plain mix): the regime where one
    batched graph replay replaces hundreds of short per-scene launches."""
    rng = np.random.default_rng(seed)
    return [plain_scene(int(rng.integers(0, 2 ** 31)), 64, 64, int(rng.integers(4, 17))) for _ in range(count)]


def batched_options() -> RenderOptions:
    return RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=True, use_prefiltering=False)


def large_scene(seed: int = 0, width: int = 1024, height: int = 1024, num_paths: int = 4096) -> Scene:
    rng = np.random.default_rng(seed)
    sc = Scene(width, height)
    sc.background = Color(1.0, 1.0, 1.0, 1.0)
    sc.filter = Filter(FilterType.BOX, 0.5)
    for i in range(num_paths):
        r = float(rng.uniform(8.0, 32.0))
        shape = Shape(PathGeometry(_closed_cubic(rng, 16, -r, r)))
        shape.transform = Mat3.rotate(float(rng.uniform(0, 2 * math.pi))).mul(
            Mat3.scale(float(rng.uniform(0.75, 1.5)), float(rng.uniform(0.75, 1.5))))
        stroked = rng.uniform() < 0.25
        if stroked:
            shape.stroke_width = float(np.float32(rng.uniform(0.5, 8.0)))
        sc.shapes.append(shape)
        cx, cy = float(rng.uniform(0, width)), float(rng.uniform(0, height))
        fill = RadialGradient((cx, cy), (2 * r, 2 * r), _stops(rng, 3))
        grp = ShapeGroup([i], fill, _solid(rng) if stroked else None)
        grp.set_shape_to_canvas(Mat3.translate(cx, cy).mul(Mat3.rotate(float(rng.uniform(0, 2 * math.pi)))))
        sc.groups.append(grp)
    return sc


def primitives_scene() -> Scene:
    """Every primitive and paint kind once on a 64x64 canvas (edge-case coverage)."""
    sc = Scene(64, 64)
    sc.background = Color(0.9, 0.9, 0.9, 1.0)
    sc.shapes.append(Shape(Circle((20.0, 20.0), 12.0)))
    e = Shape(Ellipse((44.0, 24.0), (14.0, 8.0)))
    e.stroke_width = 2.0
    sc.shapes.append(e)
    r = Shape(Rect((10.0, 36.0), (30.0, 58.0)))
    r.transform = Mat3.rotate(0.3)
    sc.shapes.append(r)
    p = Path([1, 0, 2], [(36.0, 40.0), (60.0, 30.0), (58.0, 60.0), (40.0, 62.0), (30.0, 50.0), (38.0, 46.0)],
             None, True, False)
    ps = Shape(PathGeometry(p))
    ps.stroke_width = 1.5
    sc.shapes.append(ps)
    open_path = Path([0, 0], [(4.0, 4.0), (30.0, 10.0), (60.0, 4.0)], [1.0, 3.0, 0.5], False, False)
    os_ = Shape(PathGeometry(open_path))
    os_.stroke_width = 1.0
    sc.shapes.append(os_)
    stops = [GradientStop(0.1, Color(1, 0, 0, 1)), GradientStop(0.6, Color(0, 1, 0, 0.7)),
             GradientStop(0.9, Color(0, 0, 1, 1))]
    sc.groups.append(ShapeGroup([0], LinearGradient((8.0, 8.0), (32.0, 30.0), stops), None))
    sc.groups.append(ShapeGroup([1], RadialGradient((44.0, 24.0), (14.0, 9.0), stops), Color(0.1, 0.2, 0.3, 1.0)))
    g = ShapeGroup([2, 3], Color(0.3, 0.6, 0.2, 0.6), Color(0.0, 0.0, 0.0, 0.9))
    g.fill_rule = FillRule.EVEN_ODD
    g.set_shape_to_canvas(Mat3.translate(2.0, -1.0).mul(Mat3.scale(1.05, 0.95)))
    sc.groups.append(g)
    sc.groups.append(ShapeGroup([4], None, Color(0.8, 0.1, 0.5, 1.0)))
    return sc


def styled_stroke_scene(seed: int = 0, width: int = 96, height: int = 96, num_paths: int = 12) -> Scene:
    """Stroked paths with every join and cap (the library's extension beyond the
    crate's round-only stroking)."""
    rng = np.random.default_rng(seed)
    sc = Scene(width, height)
    sc.background = Color(1.0, 1.0, 1.0, 1.0)
    sc.filter = Filter(FilterType.BOX, 0.5)
    side = float(min(width, height))
    for i in range(num_paths):
        closed = bool(rng.uniform() < 0.35)
        nseg = int(rng.integers(2, 6))
        ncp = [int(rng.integers(0, 3)) for _ in range(nseg)]
        npts = sum(c + 1 for c in ncp) + (0 if closed else 1)
        cx, cy = rng.uniform(0.2 * side, 0.8 * side, 2)
        r = rng.uniform(0.1, 0.3) * side
        pts = [(float(np.float32(cx + rng.uniform(-r, r))), float(np.float32(cy + rng.uniform(-r, r))))
               for _ in range(npts)]
        thick = None
        if rng.uniform() < 0.25:
            thick = [float(np.float32(rng.uniform(0.5, 3.0))) for _ in range(npts)]
        sh = Shape(PathGeometry(Path(ncp, pts, thick, closed, False)))
        sh.stroke_width = float(np.float32(rng.uniform(0.75, 4.0)))
        sh.stroke_join = StrokeJoin(int(rng.integers(0, 3)))
        sh.stroke_cap = StrokeCap(int(rng.integers(0, 3)))
        sh.stroke_miter_limit = float(np.float32(rng.uniform(1.0, 6.0)))
        sc.shapes.append(sh)
        fill = _solid(rng) if closed and rng.uniform() < 0.5 else None
        sc.groups.append(ShapeGroup([i], fill, _solid(rng)))
    return sc
