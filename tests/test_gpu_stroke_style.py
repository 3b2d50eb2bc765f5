"""GPU parity for stroke joins and caps other than round (the library's extension of
the crate's round-only stroking): images against the oracle (1e-5 per channel) and
render_backward gradients (same PCG32 boundary samples; 1e-4 of each array's scale),
on scenes that use every join and cap, with and without per-point thickness, through
the fused call with the fragment cache too."""
import numpy as np
import pytest

import pyoracle as orc
from dvg import BackwardOptions, DeviceGrads, Renderer, RenderOptions, synth
from dvg.scene import StrokeCap, StrokeJoin

pytestmark = pytest.mark.gpu

SEEDS = [0, 1, 2, 3]


@pytest.fixture(scope="module")
def renderer():
    r = Renderer(0)
    yield r
    r.close()


def _opts(seed):
    return RenderOptions(samples_x=2, samples_y=2, seed=seed, jitter=True, use_prefiltering=False)


@pytest.mark.parametrize("seed", SEEDS)
def test_styled_render_matches_oracle(renderer, seed):
    sc = synth.styled_stroke_scene(seed)
    img = renderer.render(sc, _opts(seed)).pixels
    ref = orc.render(sc, _opts(seed))
    assert float(np.max(np.abs(img - ref))) <= 1e-5


def test_styles_change_the_image(renderer):
    sc = synth.styled_stroke_scene(1)
    styled = renderer.render(sc, _opts(1)).pixels
    for s in sc.shapes:
        s.stroke_join, s.stroke_cap = StrokeJoin.ROUND, StrokeCap.ROUND
    rounded = renderer.render(sc, _opts(1)).pixels
    assert int((np.abs(styled - rounded).max(-1) > 1e-6).sum()) > 50


@pytest.mark.parametrize("seed", SEEDS[:2])
def test_styled_backward_matches_oracle(renderer, seed):
    sc = synth.styled_stroke_scene(seed)
    opts = _opts(seed)
    bo = BackwardOptions(boundary_samples=4000)
    d_render = np.random.default_rng(seed).standard_normal((sc.height, sc.width, 4)).astype(np.float32)
    g = renderer.render_backward(sc, opts, bo, d_render)
    _, ref = orc.render_backward(sc, opts, bo, d_render)
    for name in ("d_points", "d_paint_params", "d_shape_stroke_width", "d_thickness", "d_background"):
        a, b = g.buffers[name], ref[name]
        scale = float(np.max(np.abs(b))) if b.size else 0.0
        assert float(np.max(np.abs(a - b))) <= 1e-4 * (scale + 1e-6) + 1e-6, name


def test_styled_fused_step_uses_the_same_fragments(renderer):
    import torch

    sc = synth.styled_stroke_scene(5)
    opts = _opts(5)
    up = renderer.upload(sc)
    n = sc.width * sc.height * 4
    tgt = torch.rand(n, device="cuda")
    outs = []
    for slots in (0, 16):
        up.set_tuning(1, 4, slots)
        out = torch.empty(n, device="cuda")
        loss = torch.zeros(1, device="cuda")
        g = DeviceGrads(up.packed, "cuda")
        up.fwd_bwd_l2_device(opts, BackwardOptions(boundary_samples=3000), tgt.data_ptr(), out.data_ptr(),
                             loss.data_ptr(), g)
        torch.cuda.synchronize()
        outs.append((out.cpu().numpy(), {k: v.cpu().numpy() for k, v in g.tensors.items()}))
    assert float(np.max(np.abs(outs[0][0] - outs[1][0]))) <= 2e-6
    for k, v in outs[0][1].items():
        scale = float(np.max(np.abs(v))) if v.size else 0.0
        assert float(np.max(np.abs(outs[1][1][k] - v))) <= 1e-4 * (scale + 1e-6) + 1e-6, k
    up.close()


# ---------------------------------------------------------------- prefiltered coverage
def _pf_opts():
    return RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=False, use_prefiltering=True)


@pytest.mark.parametrize("seed", SEEDS[:2])
def test_styled_prefiltered_matches_oracle(renderer, seed):
    """Prefiltered coverage at excluded join / cap ends (the signed distance to the region's
    outer edges): image and every gradient array against the oracle."""
    sc = synth.styled_stroke_scene(seed)
    opts = _pf_opts()
    img = renderer.render(sc, opts).pixels
    ref = orc.render(sc, opts)
    assert float(np.max(np.abs(img - ref))) <= 1e-5
    for s in sc.shapes:  # the styled coverage is in use
        s.stroke_join, s.stroke_cap = StrokeJoin.ROUND, StrokeCap.ROUND
    assert float(np.max(np.abs(orc.render(sc, opts) - ref))) > 1e-2
    sc = synth.styled_stroke_scene(seed)
    d_render = np.random.default_rng(seed).standard_normal((sc.height, sc.width, 4)).astype(np.float32)
    bo = BackwardOptions(compute_translation=True)
    g = renderer.render_backward(sc, opts, bo, d_render)
    _, rb = orc.render_backward(sc, opts, bo, d_render)
    for name in rb.NAMES:
        a, b = g.buffers[name], rb[name]
        if a is None or b is None or not b.size:
            continue
        scale = float(np.max(np.abs(b)))
        assert float(np.max(np.abs(a - b))) <= 1e-4 * (scale + 1e-6) + 1e-6, name
