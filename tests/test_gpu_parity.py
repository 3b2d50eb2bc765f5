"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Images: max |gpu - oracle| <= 1e-5 per channel (same seeds, same PCG32 sample
offsets).  Gradients (same PCG32 boundary samples): per gradient array,
max |gpu - oracle| <= 1e-4 * (max |oracle| + 1e-6) + 1e-6 — only float-atomic
summation order differs.
"""
import numpy as np
import pytest

import pyoracle as orc
from dvg import BackwardOptions, Color, Renderer, RenderOptions, Rng, synth
from dvg.scene import Scene

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
GRAD_RTOL = 1e-4


@pytest.fixture(scope="module")
def renderer():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    r = Renderer(0)
    yield r
    r.close()


def _img_err(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))


def _grad_check(gpu_buf, ref_buf, names=None, rtol=GRAD_RTOL):
    worst = {}
    for n in names or gpu_buf.NAMES:
        g, r = gpu_buf[n], ref_buf[n]
        if g is None or r is None:
            continue
        scale = float(np.max(np.abs(r))) if r.size else 0.0
        err = float(np.max(np.abs(g - r))) if r.size else 0.0
        worst[n] = (err, scale)
        assert err <= rtol * (scale + 1e-6) + 1e-6, f"{n}: max err {err:.3e} vs scale {scale:.3e}"
    return worst


def test_render_plain_matches_oracle(renderer):
    sc = synth.plain_scene(0, 64, 64, 8)
    opts = synth.plain_options()
    img = renderer.render(sc, opts).pixels
    ref = orc.render(sc, opts)
    assert _img_err(img, ref) <= IMG_TOL


def test_render_mixed_matches_oracle(renderer):
    sc = synth.mixed_scene(3, 128, 128, scale=0.125, size_scale=0.25)
    opts = synth.mixed_options()
    img = renderer.render(sc, opts).pixels
    ref = orc.render(sc, opts)
    assert _img_err(img, ref) <= IMG_TOL


def test_render_no_jitter_and_filters(renderer):
    sc = synth.plain_scene(5, 48, 40, 6)
    for ft, radius in ((1, 1.0), (2, 1.5), (3, 1.0), (4, 2.0), (0, 0.0)):
        sc.filter.filter_type = ft
        sc.filter.radius = radius
        opts = RenderOptions(samples_x=3, samples_y=2, seed=7, jitter=False, use_prefiltering=False)
        img = renderer.render(sc, opts).pixels
        assert _img_err(img, orc.render(sc, opts)) <= IMG_TOL, (ft, radius)


def test_render_edge_cases(renderer):
    opts = synth.plain_options()
    empty = Scene(32, 24)
    empty.background = Color(0.2, 0.4, 0.6, 0.8)
    img = renderer.render(empty, opts).pixels
    assert np.allclose(img, np.array([0.2, 0.4, 0.6, 0.8], np.float32))
    assert renderer.render(Scene(0, 16), opts).pixels.size == 0
    sc = synth.plain_scene(2, 40, 40, 4)
    sc.background_image = np.random.default_rng(0).uniform(0, 1, (40, 40, 4)).astype(np.float32)
    assert _img_err(renderer.render(sc, opts).pixels, orc.render(sc, opts)) <= IMG_TOL


def _primitives_scene():
    return synth.primitives_scene()


def test_render_primitives_matches_oracle(renderer):
    sc = _primitives_scene()
    opts = RenderOptions(samples_x=4, samples_y=4, seed=3, jitter=True, use_prefiltering=False)
    assert _img_err(renderer.render(sc, opts).pixels, orc.render(sc, opts)) <= IMG_TOL


def _backward_case(renderer, sc, opts, bopts=None):
    bopts = bopts or BackwardOptions()
    img = orc.render(sc, opts)
    rng = np.random.default_rng(11)
    target = np.clip(img + rng.normal(0, 0.1, img.shape).astype(np.float32), 0, 1)
    d_render = (2.0 * (img - target)).astype(np.float32)
    g = renderer.render_backward(sc, opts, bopts, d_render)
    _, ref = orc.render_backward(sc, opts, bopts, d_render)
    return g.buffers, ref


def test_backward_plain_matches_oracle(renderer):
    sc = synth.plain_scene(0, 48, 48, 6)
    gpu, ref = _backward_case(renderer, sc, synth.plain_options())
    _grad_check(gpu, ref)


def test_backward_primitives_matches_oracle(renderer):
    sc = _primitives_scene()
    opts = RenderOptions(samples_x=2, samples_y=2, seed=5, jitter=True, use_prefiltering=False)
    gpu, ref = _backward_case(renderer, sc, opts, BackwardOptions(compute_translation=True))
    _grad_check(gpu, ref)


def test_backward_mixed_matches_oracle(renderer):
    sc = synth.mixed_scene(4, 96, 96, scale=0.1, size_scale=0.25)
    opts = RenderOptions(samples_x=2, samples_y=2, seed=1, jitter=True, use_prefiltering=False)
    gpu, ref = _backward_case(renderer, sc, opts)
    _grad_check(gpu, ref)


def test_backward_philox_matches_oracle(renderer):
    sc = synth.plain_scene(3, 40, 40, 5)
    b = BackwardOptions(rng=Rng.PHILOX, boundary_seed=1234, boundary_samples=5000)
    gpu, ref = _backward_case(renderer, sc, synth.plain_options(), b)
    _grad_check(gpu, ref)


def test_backward_background_image(renderer):
    sc = synth.plain_scene(2, 32, 32, 4)
    sc.background_image = np.random.default_rng(1).uniform(0, 1, (32, 32, 4)).astype(np.float32)
    gpu, ref = _backward_case(renderer, sc, synth.plain_options())
    _grad_check(gpu, ref)


# ---------------------------------------------------------------- prefiltering (the crate's default mode)
def _prefilter_opts(n=2, seed=0):
    return RenderOptions(samples_x=n, samples_y=n, seed=seed, jitter=True, use_prefiltering=True)


def test_render_prefilter_matches_oracle(renderer):
    for sc in (synth.plain_scene(1, 48, 48, 6), _primitives_scene(),
               synth.mixed_scene(6, 96, 96, scale=0.1, size_scale=0.25)):
        opts = _prefilter_opts()
        assert _img_err(renderer.render(sc, opts).pixels, orc.render(sc, opts)) <= IMG_TOL


def test_backward_prefilter_plain_matches_oracle(renderer):
    sc = synth.plain_scene(2, 40, 40, 5)
    gpu, ref = _backward_case(renderer, sc, _prefilter_opts())
    _grad_check(gpu, ref)


def test_backward_prefilter_primitives_matches_oracle(renderer):
    sc = _primitives_scene()
    gpu, ref = _backward_case(renderer, sc, _prefilter_opts(), BackwardOptions(compute_translation=True))
    _grad_check(gpu, ref)


def test_backward_prefilter_mixed_matches_oracle(renderer):
    sc = synth.mixed_scene(7, 80, 80, scale=0.08, size_scale=0.25)
    gpu, ref = _backward_case(renderer, sc, _prefilter_opts())
    _grad_check(gpu, ref)


def _reach_scene():
    """48x48 (3x3 tiles of 16 pixels), each shape ending 0.4-0.65 pixel short of a
    tile edge: prefiltered coverage (smoothstep of the distance, 1 pixel past a fill
    and stroke width + 1 past a stroke) crosses into the next tile, where the
    point-sampled tile binning does not list the group."""
    from dvg import Circle, Ellipse, Path, PathGeometry, Shape, ShapeGroup

    sc = Scene(48, 48)
    sc.background = Color(1.0, 1.0, 1.0, 1.0)
    geoms = [
        (Circle((8.0, 24.0), 7.35), 0.0),  # right edge x = 15.35, next tile from x = 16
        (Ellipse((40.0, 40.0), (7.4, 5.0)), 0.0),  # left edge x = 32.6, previous tile to x = 32
        (PathGeometry(Path([0], [(20.0, 29.45), (28.0, 29.45)], None, False, False)), 2.0),  # y + 2 + 1 > 32
    ]
    for k, (geom, sw) in enumerate(geoms):
        shape = Shape(geom)
        shape.stroke_width = sw
        sc.shapes.append(shape)
        paint = Color(0.9 * (k == 0), 0.8 * (k == 1), 0.7 * (k == 2), 1.0)
        sc.groups.append(ShapeGroup([k], None, paint) if sw > 0 else ShapeGroup([k], paint, None))
    return sc


def test_prefilter_coverage_reaches_past_tile_edges(renderer):
    """Prefiltered image and gradients where coverage crosses tile edges that the
    groups' point-sampled boxes stop short of."""
    sc = _reach_scene()
    opts = _prefilter_opts()
    ref = orc.render(sc, opts)
    # the oracle covers the pixels across each edge (the case is exercised)
    for x, y in ((16, 24), (31, 40), (24, 32)):
        assert np.max(np.abs(ref[y, x, :3] - 1.0)) > 1e-3, (x, y)
    assert _img_err(renderer.render(sc, opts).pixels, ref) <= IMG_TOL
    gpu, gref = _backward_case(renderer, sc, opts, BackwardOptions(compute_translation=True))
    _grad_check(gpu, gref)
