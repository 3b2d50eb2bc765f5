"""Signed-distance path on the GPU through the C ABI against the oracle:
render_sdf, eval_positions, the d_sdf part of render_backward (alone and together
with d_render), eval_positions_backward.  Distances: |gpu - oracle| <= 1e-5 *
(1 + |oracle|) (the device's f32 sin/cos in the ellipse solve may differ from the
host libm by an ulp); gradients: the parity bar of the other tests, 1e-4 of each
array's scale."""
import numpy as np
import pytest

import pyoracle as orc
from dvg import BackwardOptions, Renderer, RenderOptions, synth

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-4


@pytest.fixture(scope="module")
def renderer():
    r = Renderer(0)
    yield r
    r.close()


def _scenes():
    return [synth.primitives_scene(), synth.plain_scene(3, 48, 40, 6),
            synth.mixed_scene(8, 80, 72, scale=0.08, size_scale=0.25)]


def _close(a, b):
    return float(np.max(np.abs(a - b) / (1.0 + np.abs(b))))


def _grad_check(gpu, ref):
    for n in gpu.NAMES:
        g, r = gpu[n], ref[n]
        if g is None or r is None or r.size == 0:
            continue
        scale = float(np.max(np.abs(r)))
        assert float(np.max(np.abs(g - r))) <= GRAD_RTOL * (scale + 1e-6) + 1e-6, n


@pytest.mark.parametrize("opts", [RenderOptions(samples_x=2, samples_y=2, seed=1, jitter=True, use_prefiltering=False),
                                  RenderOptions(samples_x=3, samples_y=2, seed=4, jitter=True, use_prefiltering=False),
                                  RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=True, use_prefiltering=True)])
def test_render_sdf_matches_oracle(renderer, opts):
    for sc in _scenes():
        got = renderer.render_sdf(sc, opts).values
        ref = orc.render_sdf(sc, opts)
        assert got.shape == ref.shape
        assert _close(got, ref) <= 1e-5


def test_eval_positions_matches_oracle(renderer):
    rng = np.random.default_rng(3)
    for sc in _scenes():
        pos = rng.uniform(-8.0, sc.width + 8.0, (333, 2)).astype(np.float32)
        assert _close(renderer.eval_positions(sc, pos), orc.eval_positions(sc, pos)) <= 1e-5
    assert renderer.eval_positions(_scenes()[0], np.zeros((0, 2), np.float32)).size == 0


@pytest.mark.parametrize("with_render", [False, True])
def test_sdf_backward_matches_oracle(renderer, with_render):
    opts = RenderOptions(samples_x=2, samples_y=2, seed=2, jitter=True, use_prefiltering=False)
    for sc in _scenes():
        rng = np.random.default_rng(5)
        d_sdf = rng.normal(0, 1, (sc.height, sc.width)).astype(np.float32)
        bo = BackwardOptions(compute_translation=True)
        dr = None
        if with_render:
            img = orc.render(sc, opts)
            dr = rng.normal(0, 0.1, img.shape).astype(np.float32)
        g = renderer.render_backward(sc, opts, bo, dr, d_sdf).buffers
        _, ref = orc.sdf_backward(sc, opts, bo, d_sdf)
        if with_render:
            _, ref_c = orc.render_backward(sc, opts, bo, dr)
            for n in ref.NAMES:
                if ref[n] is not None and ref_c[n] is not None:
                    ref[n][...] = ref[n] + ref_c[n]
        _grad_check(g, ref)


def test_eval_positions_backward_matches_oracle(renderer):
    rng = np.random.default_rng(9)
    for sc in _scenes():
        pos = rng.uniform(-4.0, sc.width + 4.0, (500, 2)).astype(np.float32)
        d = rng.normal(0, 1, 500).astype(np.float32)
        d[::7] = 0.0
        bo = BackwardOptions(compute_translation=True)
        g = renderer.eval_positions_backward(sc, pos, None, bo, d).buffers
        _, ref = orc.eval_positions_backward(sc, pos, bo, d)
        _grad_check(g, ref)


def test_sdf_many_groups_matches_oracle(renderer):
    """200 groups: the closest-group search walks the linear BVH over group boxes."""
    sc = synth.large_scene(2, 112, 96, 200)
    opts = RenderOptions(samples_x=2, samples_y=1, seed=6, jitter=True, use_prefiltering=False)
    assert _close(renderer.render_sdf(sc, opts).values, orc.render_sdf(sc, opts)) <= 1e-5
    pos = np.random.default_rng(4).uniform(-20.0, 130.0, (400, 2)).astype(np.float32)
    assert _close(renderer.eval_positions(sc, pos), orc.eval_positions(sc, pos)) <= 1e-5
    d = np.random.default_rng(5).normal(0, 1, 400).astype(np.float32)
    bo = BackwardOptions()
    _grad_check(renderer.eval_positions_backward(sc, pos, None, bo, d).buffers,
                orc.eval_positions_backward(sc, pos, bo, d)[1])
