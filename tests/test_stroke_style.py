"""Stroke joins and caps other than round (an extension: the crate strokes every path
with round joins and caps).  Known answers on hand-worked geometry for the oracle's
restatement of the library's join / cap regions, through both the BVH and the
brute-force within tests; round joins and caps keep the crate's test."""
import pytest

import pyoracle as orc
from dvg import Color, Path, PathGeometry, Scene, Shape, ShapeGroup
from dvg.scene import StrokeCap, StrokeJoin

J, C_ = StrokeJoin, StrokeCap


def _scene(points, closed, join, cap, miter=4.0, ncp=None, radius=1.0):
    sc = Scene(32, 32)
    p = Path(ncp if ncp is not None else [0] * (len(points) - (0 if closed else 1)), list(points), None, closed, False)
    sh = Shape(PathGeometry(p))
    sh.stroke_width = radius
    sh.stroke_join, sh.stroke_cap, sh.stroke_miter_limit = join, cap, miter
    sc.shapes.append(sh)
    sc.groups.append(ShapeGroup([0], None, Color(0.0, 0.0, 0.0, 1.0)))
    return sc


def _within(sc, pt):
    a = orc.within_distance(sc, 0, pt, use_bvh=True)
    b = orc.within_distance(sc, 0, pt, use_bvh=False)
    assert a == b, f"BVH and brute-force within tests disagree at {pt}"
    return a


# Open L-shaped polyline (0,0) -> (10,0) -> (10,10), radius 1: a left turn at (10,0),
# whose outer corner is the quadrant x > 10, y < 0.
L_PTS = [(0.0, 0.0), (10.0, 0.0), (10.0, 10.0)]
CASES = [
    # point, {style: expected}
    ((-0.5, 0.0), {"round": True, "butt": False, "square": True}),     # beyond the start, on the axis
    ((-0.5, 0.9), {"round": False, "butt": False, "square": True}),    # square cap corner region
    ((-1.5, 0.0), {"round": False, "butt": False, "square": False}),   # beyond every cap
    ((5.0, 0.9), {"round": True, "butt": True, "square": True}),       # segment body
    ((5.0, 1.1), {"round": False, "butt": False, "square": False}),
    ((9.5, 0.5), {"round": True, "butt": True, "square": True}),       # inner side of the corner
]
CORNER = [
    # point, {join: expected} at the outer corner (10, 0)
    ((10.4, -0.4), {J.ROUND: True, J.BEVEL: True, J.MITER: True}),
    ((10.8, -0.8), {J.ROUND: False, J.BEVEL: False, J.MITER: True}),   # miter tip (11, -1)
    ((10.2, -0.7), {J.ROUND: True, J.BEVEL: True, J.MITER: True}),     # inside the round disc and the bevel
    ((10.2, -0.95), {J.ROUND: True, J.BEVEL: False, J.MITER: True}),   # in the disc, past the bevel edge x - y = 11
    ((11.2, -1.2), {J.ROUND: False, J.BEVEL: False, J.MITER: False}),  # past the miter tip
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_caps_known_answers(case):
    pt, want = CASES[case]
    for name, cap in (("round", C_.ROUND), ("butt", C_.BUTT), ("square", C_.SQUARE)):
        sc = _scene(L_PTS, False, J.ROUND, cap)
        assert _within(sc, pt) == want[name], (pt, name)


@pytest.mark.parametrize("case", range(len(CORNER)))
def test_joins_known_answers(case):
    pt, want = CORNER[case]
    for join, expected in want.items():
        sc = _scene(L_PTS, False, join, C_.BUTT)
        assert _within(sc, pt) == expected, (pt, join)


def test_miter_limit_falls_back_to_bevel():
    # a right angle has miter ratio sqrt(2): limit 1.2 bevels, limit 1.5 mitres
    assert not _within(_scene(L_PTS, False, J.MITER, C_.BUTT, miter=1.2), (10.8, -0.8))
    assert _within(_scene(L_PTS, False, J.MITER, C_.BUTT, miter=1.5), (10.8, -0.8))


def test_closed_path_joins_everywhere_and_ignores_caps():
    sq = [(4.0, 4.0), (14.0, 4.0), (14.0, 14.0), (4.0, 14.0)]
    for cap in (C_.BUTT, C_.SQUARE, C_.ROUND):
        # the closing vertex (4, 4) is a join too: its outer corner is (3, 3)
        assert _within(_scene(sq, True, J.MITER, cap), (3.2, 3.2))
        assert not _within(_scene(sq, True, J.BEVEL, cap), (3.2, 3.2))
        assert not _within(_scene(sq, True, J.ROUND, cap), (3.2, 3.2))
        assert _within(_scene(sq, True, J.ROUND, cap), (3.5, 3.5))


def test_curved_segments_use_their_end_tangents():
    # one cubic from (0,0) to (10,0) leaving and arriving horizontally, then a line up
    pts = [(0.0, 0.0), (3.0, 0.0), (7.0, 0.0), (10.0, 0.0), (10.0, 10.0)]
    sc_butt = _scene(pts, False, J.MITER, C_.BUTT, ncp=[2, 0])
    sc_sq = _scene(pts, False, J.MITER, C_.SQUARE, ncp=[2, 0])
    assert not _within(sc_butt, (-0.5, 0.0)) and _within(sc_sq, (-0.5, 0.0))
    assert _within(sc_butt, (10.8, -0.8))  # miter at the cubic -> line corner
    # beyond the line's end (10, 10) going up
    assert not _within(sc_butt, (10.0, 10.5)) and _within(sc_sq, (10.0, 10.5))


def test_round_style_is_the_crate_test():
    # round joins and caps: within iff the distance to the centreline is below the radius
    sc = _scene(L_PTS, False, J.ROUND, C_.ROUND)
    for pt, want in (((-0.7, 0.7), True), ((-0.75, 0.75), False), ((10.7, -0.7), True), ((10.75, -0.75), False)):
        assert _within(sc, pt) == want, pt


# ---- the edge-sampling term of styled strokes (join and cap outline edges)
def _quad_scene(pts, join, radius=2.0):
    from dvg import Filter, FilterType

    sc = Scene(40, 40)
    sc.background = Color(1.0, 1.0, 1.0, 1.0)
    sc.filter = Filter(FilterType.BOX, 0.5)
    sh = Shape(PathGeometry(Path([0] * len(pts), [tuple(map(float, p)) for p in pts], None, True, False)))
    sh.stroke_width = radius
    sh.stroke_join, sh.stroke_miter_limit = join, 6.0
    sc.shapes.append(sh)
    sc.groups.append(ShapeGroup([0], None, Color(0.1, 0.2, 0.8, 1.0)))
    return sc


def _edge_grads(sc, n_samples, seeds, base=100):
    """Mean and standard error over seeds of the edge term alone (interior pass off),
    with d_render = 1 on the colour channels (the loss is the summed colour)."""
    import os

    import numpy as np

    from dvg import BackwardOptions, RenderOptions

    w = np.ones((sc.height, sc.width, 4), np.float32)
    w[..., 3] = 0.0
    opts = RenderOptions(samples_x=2, samples_y=2, seed=1, jitter=True, use_prefiltering=False)
    pts, rad = [], []
    for s in range(seeds):
        _, b = orc.render_backward(sc, opts, BackwardOptions(boundary_samples=n_samples, boundary_seed=base + s), w,
                                   passes=2, threads=os.cpu_count() or 1)
        pts.append(np.asarray(b["d_points"], np.float64).copy())
        rad.append(float(b["d_shape_stroke_width"][0]))
    pts, rad = np.stack(pts), np.asarray(rad)
    return pts.mean(0), rad.mean(), rad.std(ddof=1) / np.sqrt(seeds)


DELTA = (0.1 - 1.0) + (0.2 - 1.0) + (0.8 - 1.0)  # colour minus white background, summed


@pytest.mark.parametrize("join", [J.BEVEL, J.MITER])
def test_join_edges_give_the_exact_radius_gradient(join):
    # square of side L around its centreline, radius r: stroke area 8 L r - 2 r^2 (bevel), 8 L r (miter)
    L, r, c = 16.0, 2.0, 12.3
    sc = _quad_scene([(c, c), (c + L, c), (c + L, c + L), (c, c + L)], join, r)
    _, g, se = _edge_grads(sc, 100000, 12)
    exact = DELTA * (8 * L - 4 * r if join == J.BEVEL else 8 * L)
    assert abs(g - exact) <= 0.005 * abs(exact) + 4 * se, (g, exact, se)


def test_mitred_vertex_gradients_match_the_area_derivative():
    import numpy as np

    r = 2.0
    P = np.array([(11.3, 12.1), (28.4, 10.7), (29.2, 27.9), (12.6, 26.8)], np.float64)

    def offset_area(Q, s):  # mitred offset polygon (every join within the limit here)
        out = []
        for i in range(len(Q)):
            a, v, b = Q[i - 1], Q[i], Q[(i + 1) % len(Q)]
            d0, d1 = (v - a) / np.linalg.norm(v - a), (b - v) / np.linalg.norm(b - v)
            a0, a1 = v + s * np.array([d0[1], -d0[0]]), v + s * np.array([d1[1], -d1[0]])
            cr = d0[0] * d1[1] - d0[1] * d1[0]
            out.append(a0 + ((a1 - a0)[0] * d1[1] - (a1 - a0)[1] * d1[0]) / cr * d0)
        x, y = np.array(out).T
        return 0.5 * abs(np.dot(x, np.roll(y, -1)) - np.dot(y, np.roll(x, -1)))

    def stroke_area(Q):
        return abs(offset_area(Q, r) - offset_area(Q, -r))

    g, _, _ = _edge_grads(_quad_scene(P, J.MITER, r), 100000, 12)
    h = 1e-5
    for i in range(4):
        for c in range(2):
            a, b = P.copy(), P.copy()
            a[i, c] += h
            b[i, c] -= h
            exact = DELTA * (stroke_area(a) - stroke_area(b)) / (2 * h)
            assert abs(g[2 * i + c] - exact) <= 0.02 * abs(exact) + 0.05, (i, c, g[2 * i + c], exact)


def test_boundary_sample_count_keeps_the_expectation():
    # the crate draws W*H*spp edge samples; fewer (here W*H) must estimate the same gradient
    L, r, c = 16.0, 2.0, 12.3
    sc = _quad_scene([(c, c), (c + L, c), (c + L, c + L), (c, c + L)], J.BEVEL, r)
    _, g, se = _edge_grads(sc, 40 * 40, 48, base=7000)
    exact = DELTA * (8 * L - 4 * r)
    assert abs(g - exact) <= 4 * se + 0.005 * abs(exact), (g, exact, se)
