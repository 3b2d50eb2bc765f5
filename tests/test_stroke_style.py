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
