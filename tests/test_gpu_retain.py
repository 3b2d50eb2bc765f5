"""Retained render (dvg_context_set_retain): dvg_render keeps its prepared scene,
weight image and fragment codes; a dvg_render_backward of the same description and
options reuses them and gives the same gradients as a fresh backward (1e-4 of
scale: float summation order), while any change (one point moved, other options, a
render of another scene in between) falls back to the full backward."""
import numpy as np
import pytest

from dvg import BackwardOptions, Renderer, RenderOptions, synth
from dvg.abi import pack_scene

pytestmark = pytest.mark.gpu


def _grad_arrays(g):
    return {k: v.copy() for k, v in g.buffers.arrays.items() if v is not None}


def _close(a, b):
    for k in a:
        scale = float(np.max(np.abs(b[k]))) if b[k].size else 0.0
        assert float(np.max(np.abs(a[k] - b[k]))) <= 1e-4 * (scale + 1e-6) + 1e-6, k


def _fresh(r, sc, opts, bo, d_render):
    r.set_retain(False)
    g = r.render_backward(sc, opts, bo, d_render)
    r.set_retain(True)
    return _grad_arrays(g)


def _weights_launched(r):
    return "weights" in r.profile(True)


@pytest.mark.parametrize("prefilter", [False, True])
def test_backward_after_render_reuses_and_matches(prefilter):
    r = Renderer(0)
    try:
        sc = synth.mixed_scene(3, 96, 80, scale=0.1, size_scale=0.3)
        opts = RenderOptions(samples_x=2, samples_y=2, seed=4, jitter=not prefilter, use_prefiltering=prefilter)
        bo = BackwardOptions(boundary_samples=3000)
        rng = np.random.default_rng(0)
        d_render = rng.standard_normal((80, 96, 4)).astype(np.float32)
        ref = _fresh(r, sc, opts, bo, d_render)
        r.set_profiling(True)
        packed = pack_scene(sc)
        img = r.render(sc, opts, packed=packed).pixels
        r.profile(True)
        g = _grad_arrays(r.render_backward(sc, opts, bo, d_render, packed=packed))
        assert not _weights_launched(r), "the backward did not reuse the retained render"
        _close(g, ref)
        # a second backward on the same render reuses it again
        g2 = _grad_arrays(r.render_backward(sc, opts, bo, d_render))
        assert not _weights_launched(r)
        _close(g2, ref)
        r.set_retain(False)
        img0 = r.render(sc, opts).pixels
        assert float(np.max(np.abs(img - img0))) <= 2e-6
    finally:
        r.close()


def test_changes_fall_back_to_a_full_backward():
    r = Renderer(0)
    try:
        sc = synth.plain_scene(8, 64, 48, 6)
        moved = synth.plain_scene(8, 64, 48, 6)
        p = moved.shapes[2].geometry.path
        x, y = p.points[1]
        p.points[1] = (x + 0.75, y)
        opts = RenderOptions(samples_x=2, samples_y=2, seed=1, jitter=True, use_prefiltering=False)
        other = RenderOptions(samples_x=2, samples_y=2, seed=2, jitter=True, use_prefiltering=False)
        bo = BackwardOptions(boundary_samples=2000)
        d_render = np.random.default_rng(1).standard_normal((48, 64, 4)).astype(np.float32)
        r.set_profiling(True)
        # another description
        r.render(sc, opts)
        r.profile(True)
        g = _grad_arrays(r.render_backward(moved, opts, bo, d_render))
        assert _weights_launched(r)
        _close(g, _fresh(r, moved, opts, bo, d_render))
        # other options
        r.render(sc, opts)
        r.profile(True)
        g = _grad_arrays(r.render_backward(sc, other, bo, d_render))
        assert _weights_launched(r)
        _close(g, _fresh(r, sc, other, bo, d_render))
        # a render of another scene in between
        r.render(sc, opts)
        up = r.upload(moved)
        up.render_host(opts)
        r.profile(True)
        g = _grad_arrays(r.render_backward(sc, opts, bo, d_render))
        assert _weights_launched(r)
        _close(g, _fresh(r, sc, opts, bo, d_render))
        up.close()
    finally:
        r.close()
