"""The crate's own known-answer tests, restated against the CPU oracle.

These pin the oracle's distance / winding / flattening arithmetic to the only
golden values the reference ships: src/distance/tests.rs:7-136 and
src/geometry.rs:505-520.
"""
import math

import pyoracle as orc
from dvg.scene import (Circle, Color, FillRule, Path, PathGeometry, PathSegment, Rect, Scene, Shape,
                       ShapeGroup)


def test_compute_distance_circle():  # src/distance/tests.rs:7-26
    scene = Scene(100, 100)
    scene.shapes.append(Shape(Circle((50.0, 50.0), 10.0)))
    scene.groups.append(ShapeGroup([0], Color.opaque(1.0, 0.0, 0.0), None))
    hit = orc.compute_distance(scene, 0, (70.0, 50.0), math.inf)
    assert hit is not None
    assert abs(hit["distance"] - 10.0) < 1.0e-3


def test_within_distance_path_stroke():  # src/distance/tests.rs:28-51
    scene = Scene(100, 100)
    path = Path.from_segments([PathSegment.MoveTo((10.0, 10.0)), PathSegment.LineTo((90.0, 10.0))])
    path.is_closed = False
    shape = Shape(PathGeometry(path))
    shape.stroke_width = 4.0
    scene.shapes.append(shape)
    group = ShapeGroup([0], None, Color.opaque(0.0, 0.0, 0.0))
    group.fill_rule = FillRule.NON_ZERO
    scene.groups.append(group)
    assert orc.within_distance(scene, 0, (50.0, 12.0))
    assert not orc.within_distance(scene, 0, (50.0, 20.0))


def test_bvh_compute_distance_matches_linear():  # src/distance/tests.rs:53-82
    scene = Scene(100, 100)
    scene.shapes.append(Shape(Circle((20.0, 40.0), 8.0)))
    scene.shapes.append(Shape(Rect((60.0, 60.0), (80.0, 80.0))))
    scene.groups.append(ShapeGroup([0, 1], Color.opaque(1.0, 0.0, 0.0), None))
    linear = orc.compute_distance(scene, 0, (30.0, 40.0), math.inf, use_bvh=False)
    accel = orc.compute_distance(scene, 0, (30.0, 40.0), math.inf, use_bvh=True)
    assert linear is not None and accel is not None
    assert abs(linear["distance"] - accel["distance"]) < 1.0e-3
    assert linear["shape_index"] == accel["shape_index"]


def test_bvh_within_distance_matches_linear():  # src/distance/tests.rs:84-104
    scene = Scene(100, 100)
    shape = Shape(Rect((10.0, 10.0), (30.0, 30.0)))
    shape.stroke_width = 5.0
    scene.shapes.append(shape)
    scene.groups.append(ShapeGroup([0], None, Color.opaque(0.0, 0.0, 0.0)))
    for pt in ((32.0, 20.0), (50.0, 20.0)):
        assert orc.within_distance(scene, 0, pt) == orc.within_distance(scene, 0, pt, use_bvh=True)
    assert orc.within_distance(scene, 0, (32.0, 20.0))
    assert not orc.within_distance(scene, 0, (50.0, 20.0))


def test_bvh_path_distance_matches_linear():  # src/distance/tests.rs:106-136
    scene = Scene(120, 120)
    path = Path.from_segments([
        PathSegment.MoveTo((20.0, 20.0)),
        PathSegment.QuadTo((60.0, 80.0), (100.0, 20.0)),
        PathSegment.CubicTo((90.0, 90.0), (30.0, 90.0), (20.0, 20.0)),
    ])
    scene.shapes.append(Shape(PathGeometry(path)))
    scene.groups.append(ShapeGroup([0], Color(0.2, 0.3, 0.4, 1.0), None))
    linear = orc.compute_distance(scene, 0, (60.0, 40.0), math.inf, use_bvh=False)
    accel = orc.compute_distance(scene, 0, (60.0, 40.0), math.inf, use_bvh=True)
    assert linear is not None and accel is not None
    assert abs(linear["distance"] - accel["distance"]) < 1.0e-3
    assert linear["shape_index"] == accel["shape_index"]


def test_flatten_quadratic_produces_segments():  # src/geometry.rs:509-519
    scene = Scene(10, 10)
    path = Path.from_segments([PathSegment.MoveTo((0.0, 0.0)), PathSegment.QuadTo((0.5, 1.0), (1.0, 0.0))])
    scene.shapes.append(Shape(PathGeometry(path)))
    segs = orc.flatten(scene, 0, 0.01)
    assert len(segs) > 0
    assert tuple(segs[0][:2]) == (0.0, 0.0)
    assert tuple(segs[-1][2:]) == (1.0, 0.0)
