"""Prefiltered coverage of strokes with joins and caps other than round (an extension:
the crate's prefiltered stroke is round, smoothstep(|d| + sw) - smoothstep(|d| - sw),
src/backward/sampling.rs:240-260).  Where the closest point is a segment end that the
point-sampled stroke excludes, the coverage is smoothstep(s + 2 sw) - smoothstep(s)
with s the signed distance to the join / cap region's outer edges.

Known answers on hand-worked geometry (1x1 spp, box r=0.5: a pixel is its centre's
coverage, alpha = w on a transparent background), then the oracle's adjoint of that
coverage against central finite differences of its own image (points, stroke widths,
shape and group transform entries, under rotations and translations).
"""
import numpy as np
import pytest

import pyoracle as orc
from dvg import BackwardOptions, Color, Mat3, Path, PathGeometry, RenderOptions, Scene, Shape, ShapeGroup
from dvg.abi import pack_scene
from dvg.scene import StrokeCap, StrokeJoin

J, C_ = StrokeJoin, StrokeCap
ONE = RenderOptions(samples_x=1, samples_y=1, seed=0, jitter=False, use_prefiltering=True)


def _smooth(x):
    t = min(max((x + 1.0) * 0.5, 0.0), 1.0)
    return t * t * (3.0 - 2.0 * t)


def _w(s, sw):
    return _smooth(s + 2.0 * sw) - _smooth(s)


def _stroke(sc, points, closed, join, cap, sw, miter=4.0):
    p = Path([0] * (len(points) - (0 if closed else 1)), list(points), None, closed, False)
    sh = Shape(PathGeometry(p))
    sh.stroke_width = sw
    sh.stroke_join, sh.stroke_cap, sh.stroke_miter_limit = join, cap, miter
    sc.shapes.append(sh)
    sc.groups.append(ShapeGroup([len(sc.shapes) - 1], None, Color(0.0, 0.0, 0.0, 1.0)))
    return sh


def _alpha(sc, x, y):
    return float(orc.render(sc, ONE)[y, x, 3])


@pytest.mark.parametrize("cap,expect", [
    # line (8, 16.5) -> (24, 16.5), sw 2; pixel centres at x + 0.5 beyond the end x = 24
    (C_.BUTT, {24: _w(0.5, 2.0), 25: 0.0}),                       # flat end: s = distance past it
    (C_.SQUARE, {24: _w(-1.5, 2.0), 25: _w(-0.5, 2.0), 26: _w(0.5, 2.0), 27: 0.0}),  # box to x = 26
    (C_.ROUND, {24: _smooth(0.5 + 2.0) - _smooth(0.5 - 2.0), 25: _smooth(1.5 + 2.0) - _smooth(1.5 - 2.0)}),
])
def test_caps_known_answers(cap, expect):
    sc = Scene(40, 32)
    _stroke(sc, [(8.0, 16.5), (24.0, 16.5)], False, J.ROUND, cap, 2.0)
    for x, w in expect.items():
        assert _alpha(sc, x, 16) == pytest.approx(w, abs=2e-6), (cap, x)
    if cap == C_.BUTT:  # off the axis, still past the end: distance to the flat end line
        assert _alpha(sc, 24, 17) == pytest.approx(_w(0.5, 2.0), abs=2e-6)


@pytest.mark.parametrize("join,expect", [
    # A (6, 20) -> V (20, 20) -> B (20, 6), sw 3: outer corner towards +x, +y
    (J.BEVEL, {(21, 21): _w(0.0, 3.0), (22, 22): 0.0}),            # bevel edge x + y = 43
    (J.MITER, {(21, 21): _w(-1.5, 3.0), (22, 22): _w(-0.5, 3.0), (23, 23): _w(2 ** 0.5 / 2, 3.0)}),  # tip (23, 23)
    (J.ROUND, {(21, 21): _smooth(1.5 * 2 ** 0.5 + 3.0) - _smooth(1.5 * 2 ** 0.5 - 3.0)}),
])
def test_joins_known_answers(join, expect):
    sc = Scene(32, 32)
    _stroke(sc, [(6.0, 20.0), (20.0, 20.0), (20.0, 6.0)], False, join, C_.ROUND, 3.0)
    for (x, y), w in expect.items():
        assert _alpha(sc, x, y) == pytest.approx(w, abs=2e-6), (join, x, y)


def test_reversal_ends_flat_and_straight_join_stays_round():
    # a reversal at V = (24, 16.5) (out and straight back): both bodies end flat at V
    sc = Scene(40, 32)
    _stroke(sc, [(8.0, 16.5), (24.0, 16.5), (10.0, 16.5)], False, J.MITER, C_.ROUND, 2.0)
    assert _alpha(sc, 24, 16) == pytest.approx(_w(0.5, 2.0), abs=2e-6)
    # a straight join at V = (16.5, 16.5): the bodies meet, the round formula holds
    sc = Scene(40, 32)
    _stroke(sc, [(8.0, 16.5), (16.5, 16.5), (24.0, 16.5)], False, J.BEVEL, C_.ROUND, 2.5)
    assert _alpha(sc, 16, 19) == pytest.approx(_smooth(3.0 + 2.5) - _smooth(3.0 - 2.5), abs=2e-6)


def test_miter_limit_falls_back_to_bevel():
    # a right angle has miter ratio sqrt(2): limit 1.2 bevels
    sc = Scene(32, 32)
    _stroke(sc, [(6.0, 20.0), (20.0, 20.0), (20.0, 6.0)], False, J.MITER, C_.ROUND, 3.0, miter=1.2)
    assert _alpha(sc, 22, 22) == pytest.approx(0.0, abs=2e-6)


def _styled_scene():
    """40x40: an open polyline with a miter join, a bevel join and square / butt ends, and
    a closed mitred triangle, rotated and translated about the canvas centre."""
    sc = Scene(40, 40)
    sc.background = Color(0.9, 0.85, 0.8, 1.0)
    a = _stroke(sc, [(6.0, 30.0), (16.0, 12.0), (24.0, 27.0), (34.0, 8.0)], False, J.MITER, C_.SQUARE, 2.2, 6.0)
    b = _stroke(sc, [(8.0, 6.0), (30.0, 18.0), (12.0, 34.0)], True, J.BEVEL, C_.BUTT, 1.6)
    sc.groups[0].stroke = Color(0.2, 0.5, 0.9, 0.8)
    sc.groups[1].stroke = Color(0.8, 0.3, 0.1, 0.7)
    c = sc.width / 2.0
    for i, s in enumerate((a, b)):
        s.transform = Mat3.translate(c, c).mul(Mat3.rotate(0.2 * (i + 1))).mul(Mat3.translate(-c, -c))
        sc.groups[i].set_shape_to_canvas(Mat3.translate(0.7 - 0.4 * i, -0.5 + 0.3 * i))
    return sc


def test_styled_coverage_differs_from_round():
    sc = _styled_scene()
    opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=False, use_prefiltering=True)
    styled = orc.render(sc, opts)
    for s in sc.shapes:
        s.stroke_join, s.stroke_cap = J.ROUND, C_.ROUND
    rnd = orc.render(sc, opts)
    diff = np.abs(styled - rnd).max(-1)
    assert diff.max() > 0.2 and (diff > 1e-3).sum() > 30


def _params(sc):
    packed = pack_scene(sc)
    out = []
    for si, shp in enumerate(sc.shapes):
        out.append(("d_shape_stroke_width", si, lambda s=shp: s.stroke_width,
                    lambda v, s=shp: setattr(s, "stroke_width", v), 1e-3))
        base = packed.path_point_offset[si]
        for k in range(len(shp.geometry.path.points)):
            for ci in range(2):
                def get(path=shp.geometry.path, k=k, ci=ci):
                    return path.points[k][ci]

                def put(v, path=shp.geometry.path, k=k, ci=ci):
                    p = list(path.points[k])
                    p[ci] = v
                    path.points[k] = tuple(p)
                out.append(("d_points", 2 * (base + k) + ci, get, put, 1e-3))
        for k in range(6):
            h = 1e-3 if k in (2, 5) else 3e-5

            def sget(s=shp, k=k):
                return float(s.transform.m.reshape(-1)[k])

            def sput(v, s=shp, k=k):
                m = s.transform.m.reshape(-1).copy()
                m[k] = v
                s.transform = Mat3(m)
            out.append(("d_shape_transform", 9 * si + k, sget, sput, h))
            g = sc.groups[si]

            def gget(g=g, k=k):
                return float(g.shape_to_canvas.m.reshape(-1)[k])

            def gput(v, g=g, k=k):
                m = g.shape_to_canvas.m.reshape(-1).copy()
                m[k] = v
                g.set_shape_to_canvas(Mat3(m))
            out.append(("d_group_transform", 9 * si + k, gget, gput, h))
    return out


def test_styled_prefiltered_gradients_match_fd():
    """Central differences of the oracle's image against its adjoint.  Bars: points and
    transforms 5e-3 of the array's scale (the round prefiltered strokes' measured floor
    is 1e-3-3e-3 on the same kind of scene, from f32 rendering), stroke widths 2e-3.
    Steps: 1e-3 on points and translations, 3e-5 on the linear entries.  The join and cap
    distances have kinks (where the closest outer edge switches, and on the normals that
    bound an excluded end) and larger steps carry one across a sample: the mitred vertex's
    x at 2.5e-3 (measured 5.5e-2 of the scale; 1e-4-5e-4 for steps of 2e-4 to 1e-3), the
    first group's second-row linear entries at 1e-4 (3.4e-2 of the scale; 3e-4 at 3e-5)."""
    sc = _styled_scene()
    opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=False, use_prefiltering=True)
    img = orc.render_differentiated(sc, opts)
    rng = np.random.default_rng(3)
    target = np.clip(img + rng.normal(0, 0.1, img.shape).astype(np.float32), 0, 1)
    dr = (2.0 * (img - target)).astype(np.float32)
    grads = orc.render_backward(sc, opts, BackwardOptions(boundary_samples=1), dr)[1]
    dr64 = dr.astype(np.float64)
    fd = {}
    for name, idx, get, put, h in _params(sc):
        v = get()
        hp, hm = float(np.float32(v + h)), float(np.float32(v - h))
        put(hp)
        lp = float(np.sum(orc.render_differentiated(sc, opts).astype(np.float64) * dr64))
        put(hm)
        lm = float(np.sum(orc.render_differentiated(sc, opts).astype(np.float64) * dr64))
        put(v)
        fd.setdefault(name, []).append((idx, (lp - lm) / (hp - hm)))
    for name, pairs in fd.items():
        g = np.asarray(grads[name], np.float64)
        idx = np.array([i for i, _ in pairs])
        f = np.array([x for _, x in pairs])
        scale = float(np.max(np.abs(g[idx])))
        err = float(np.max(np.abs(g[idx] - f)))
        rtol = 2e-3 if name == "d_shape_stroke_width" else 5e-3
        assert scale > 0.0, name
        assert err <= rtol * scale + 1e-5, f"{name}: max |analytic - FD| {err:.3e}, scale {scale:.3e}"
