"""Signed-distance path on the CPU oracle: the adjoint of eval_positions
(render_backward_positions, src/backward/render.rs:213-265) against central finite
differences of eval_positions itself (f64 sums of f32 distances, h = 1e-2: the
distances are smooth at that scale away from medial axes, while smaller steps hit
the f32 rounding of 64 distances of tens of pixels), on one-shape scenes.  Bar: per
gradient array, 1e-3 of the gradient scale.

The ellipse centre is left out: the crate's ellipse closest-point adjoint
(src/backward/distance.rs:479-561) adds the centre's direct term only in its
degenerate branches, so in the general case its centre gradient of the distance is
~0 where the true one is not (measured here: 1e-6 against ~5).  The oracle and the
CUDA path keep that arithmetic (parity first)."""
import numpy as np
import pytest

from dvg import BackwardOptions, Color, Mat3, Scene, Shape, ShapeGroup
from dvg.abi import pack_scene
from dvg.scene import Circle, Ellipse, Path, PathGeometry, Rect


def _scene(kind):
    sc = Scene(64, 64)
    if kind == "circle":
        sh = Shape(Circle((30.0, 34.0), 13.0))
    elif kind == "rect":
        sh = Shape(Rect((14.0, 18.0), (44.0, 40.0)))
        sh.transform = Mat3.rotate(0.2)
    elif kind == "ellipse":
        sh = Shape(Ellipse((32.0, 30.0), (16.0, 9.0)))
    else:  # open quadratic + line path, stroked
        sh = Shape(PathGeometry(Path([1, 0], [(6.0, 40.0), (30.0, 4.0), (52.0, 30.0), (60.0, 58.0)], None, False,
                                     False)))
        sh.stroke_width = 2.0
    sc.shapes.append(sh)
    g = ShapeGroup([0], Color(0.5, 0.2, 0.1, 1.0) if kind != "path" else None,
                   Color(0, 0, 0, 1) if kind == "path" else None)
    g.set_shape_to_canvas(Mat3.translate(1.5, -0.5))
    sc.groups.append(g)
    return sc


def _params(sc):
    sh = sc.shapes[0]
    geo = sh.geometry
    out = []
    if isinstance(geo, Circle):
        out += [("d_shape_params", 0, geo, "center", 0), ("d_shape_params", 1, geo, "center", 1),
                ("d_shape_params", 2, geo, "radius", None)]
    elif isinstance(geo, Rect):
        out += [("d_shape_params", k, geo, f, c) for k, (f, c) in enumerate((("min", 0), ("min", 1), ("max", 0),
                                                                           ("max", 1)))]
    elif isinstance(geo, Ellipse):
        out += [("d_shape_params", 2, geo, "radius", 0), ("d_shape_params", 3, geo, "radius", 1)]
    else:
        for k in range(len(geo.path.points)):
            for c in range(2):
                out.append(("d_points", 2 * k + c, geo.path, ("points", k), c))
    return out


def _get(obj, field, c):
    if isinstance(field, tuple):
        return getattr(obj, field[0])[field[1]][c]
    v = getattr(obj, field)
    return v if c is None else v[c]


def _put(obj, field, c, val):
    if isinstance(field, tuple):
        lst = getattr(obj, field[0])
        p = list(lst[field[1]])
        p[c] = val
        lst[field[1]] = tuple(p)
        return
    if c is None:
        setattr(obj, field, val)
    else:
        p = list(getattr(obj, field))
        p[c] = val
        setattr(obj, field, tuple(p))


@pytest.mark.parametrize("kind", ["circle", "rect", "ellipse", "path"])
def test_positions_adjoint_matches_fd(kind):
    import pyoracle

    sc = _scene(kind)
    rng = np.random.default_rng(7)
    pos = rng.uniform(2.0, 62.0, (64, 2)).astype(np.float32)
    d = rng.uniform(0.5, 1.5, 64).astype(np.float32)
    _, buf = pyoracle.eval_positions_backward(sc, pos, BackwardOptions(), d)
    worst = {}
    for name, idx, obj, field, c in _params(sc):
        v = _get(obj, field, c)
        h = 1e-2
        hp, hm = float(np.float32(v + h)), float(np.float32(v - h))
        _put(obj, field, c, hp)
        lp = float(np.sum(pyoracle.eval_positions(sc, pos).astype(np.float64) * d))
        _put(obj, field, c, hm)
        lm = float(np.sum(pyoracle.eval_positions(sc, pos).astype(np.float64) * d))
        _put(obj, field, c, v)
        worst.setdefault(name, []).append((float(buf[name][idx]), (lp - lm) / (hp - hm)))
    for name, pairs in worst.items():
        a = np.array([x for x, _ in pairs])
        f = np.array([y for _, y in pairs])
        scale = float(np.max(np.abs(a)))
        assert scale > 0
        assert float(np.max(np.abs(a - f))) <= 1e-3 * scale + 1e-4, (kind, name, a, f)
    assert pack_scene(sc) is not None
