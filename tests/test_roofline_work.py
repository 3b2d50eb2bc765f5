"""The committed forward-pass work counts (profiles/roofline_work.json, read by
bench.py for the compute roofline) equal a fresh brute-force count by the oracle's
counting build, and the operation counts of single tests match hand-counted
straight-line arithmetic."""
import json
import os

import pytest

import pyoracle as orc
from dvg import Circle, Color, Path, PathGeometry, RenderOptions, Scene, Shape, ShapeGroup

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name", ["plain", "adjoint", "mixed"])
def test_committed_counts_are_current(name):
    import count_work

    with open(os.path.join(ROOT, "profiles", "roofline_work.json")) as f:
        committed = json.load(f)["workloads"][name]
    assert count_work.count(name) == committed


def _one_sample_scene(shape, fill=True, stroke=False):
    sc = Scene(1, 1)
    sc.shapes.append(shape)
    c = Color(0.5, 0.5, 0.5, 1.0)
    sc.groups.append(ShapeGroup([0], c if fill else None, c if stroke else None))
    return sc


def test_single_test_operation_counts():
    # one sample at (0.5, 0.5): no jitter, 1x1 spp
    opts = RenderOptions(samples_x=1, samples_y=1, seed=0, jitter=False, use_prefiltering=False)
    # a closed polyline: every line test costs dy (1), + t (2), + tp (4) operations
    line = Path([0, 0, 0], [(2.0, -1.0), (2.0, 2.0), (-3.0, 2.0)], None, True, False)
    n, f = orc.count_work(_one_sample_scene(Shape(PathGeometry(line))), opts)["fill_line"]
    assert n >= 1 and n <= f <= 7 * n
    # a circle containing the sample: the squared-distance test, 6 operations
    w = orc.count_work(_one_sample_scene(Shape(Circle((0.0, 0.0), 3.0))), opts)
    assert w["fill_circle"] == (1, 6)
    # its stroke test: |p - c| - |r|, 7 operations
    s = Shape(Circle((0.0, 0.0), 3.0))
    s.stroke_width = 4.0
    w = orc.count_work(_one_sample_scene(s, fill=False, stroke=True), opts)
    assert w["stroke_circle"] == (1, 7)
