"""GPU parity of the gradient-paint adjoint (backward/paint.rs:91-277) against the oracle.

The interior adjoint sums a gradient paint's terms (stop colours, stop offsets, paint
parameters) over a warp when all of the warp's contributing samples fall in one stop
interval, and adds them per sample otherwise.  These scenes cover both: large shapes
with two wide stops (whole warps in one interval), many narrow stops (warps straddling
several intervals), and stops that start late and end early (samples before the first
and after the last stop), in plain and prefiltered rendering.  Same tolerance as the
other gradient parity tests: max |gpu - oracle| <= 1e-4 * (max |oracle| + 1e-6) + 1e-6
per gradient array (only the float summation order differs).
"""
import numpy as np
import pytest

import pyoracle as orc
from dvg import BackwardOptions, Color, Renderer, RenderOptions
from dvg.scene import (Circle, Ellipse, GradientStop, LinearGradient, Mat3, Path, PathGeometry, RadialGradient,
                       Rect, Scene, Shape, ShapeGroup)

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-4


@pytest.fixture(scope="module")
def renderer():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    r = Renderer(0)
    yield r
    r.close()


def _stops(offsets, seed):
    rng = np.random.default_rng(seed)
    return [GradientStop(float(o), Color(*rng.uniform(0.05, 1.0, 4).astype(np.float32).tolist())) for o in offsets]


def gradient_scene() -> Scene:
    sc = Scene(80, 64)
    sc.background = Color(0.95, 0.95, 0.9, 1.0)
    sc.shapes.append(Shape(Rect((2.0, 2.0), (78.0, 40.0))))
    sc.shapes.append(Shape(Circle((40.0, 36.0), 26.0)))
    e = Shape(Ellipse((60.0, 48.0), (18.0, 12.0)))
    e.transform = Mat3.rotate(0.4)
    sc.shapes.append(e)
    p = Path([2, 1], [(4.0, 60.0), (20.0, 20.0), (50.0, 70.0), (70.0, 30.0), (76.0, 58.0), (60.0, 62.0)],
             None, False, False)
    ps = Shape(PathGeometry(p))
    ps.stroke_width = 3.0
    sc.shapes.append(ps)
    # two wide stops: most warps lie in one interval
    sc.groups.append(ShapeGroup([0], LinearGradient((0.0, 0.0), (80.0, 10.0), _stops([0.0, 1.0], 1)), None))
    # many narrow stops: warps straddle intervals
    sc.groups.append(ShapeGroup([1], RadialGradient((40.0, 36.0), (26.0, 20.0),
                                                    _stops([0.0, 0.08, 0.11, 0.3, 0.31, 0.55, 0.7, 1.0], 2)), None))
    # stops that start late and end early: samples before the first and after the last stop
    sc.groups.append(ShapeGroup([2], LinearGradient((45.0, 40.0), (75.0, 56.0), _stops([0.35, 0.5, 0.65], 3)), None))
    sc.groups.append(ShapeGroup([3], None, RadialGradient((40.0, 45.0), (30.0, 30.0), _stops([0.2, 0.9], 4))))
    return sc


def _check(gpu, ref):
    for n in ("d_paint_params", "d_stop_offsets", "d_stop_colors", "d_points", "d_shape_params",
              "d_shape_transform", "d_group_transform", "d_filter_radius", "d_background"):
        g, r = gpu[n], ref[n]
        if g is None or r is None or not r.size:
            continue
        scale = float(np.max(np.abs(r)))
        err = float(np.max(np.abs(g - r)))
        assert err <= GRAD_RTOL * (scale + 1e-6) + 1e-6, f"{n}: max err {err:.3e} vs scale {scale:.3e}"


@pytest.mark.parametrize("prefilter", [False, True])
@pytest.mark.parametrize("spp", [2, 4])
def test_gradient_paint_adjoint_matches_oracle(renderer, prefilter, spp):
    sc = gradient_scene()
    opts = RenderOptions(samples_x=spp, samples_y=spp, seed=9, jitter=True, use_prefiltering=prefilter)
    bopts = BackwardOptions()
    img = orc.render(sc, opts)
    rng = np.random.default_rng(5)
    target = np.clip(img + rng.normal(0, 0.15, img.shape).astype(np.float32), 0, 1)
    d_render = (2.0 * (img - target)).astype(np.float32)
    g = renderer.render_backward(sc, opts, bopts, d_render)
    _, ref = orc.render_backward(sc, opts, bopts, d_render)
    assert np.any(ref["d_stop_colors"] != 0) and np.any(ref["d_stop_offsets"] != 0)
    _check(g.buffers, ref)
