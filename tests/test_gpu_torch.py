"""torch.autograd bridge (dvg.torch_ops.render): the image equals Renderer.render and
the gradients torch computes for (points, paint_params) equal render_backward's
with the same adjoint (same PCG32 boundary samples; parity bar 1e-4 of scale)."""
import numpy as np
import pytest
import torch

from dvg import BackwardOptions, Renderer, RenderOptions, synth
from dvg.torch_ops import render, scene_tensors

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prefilter", [False, True])
def test_autograd_matches_render_backward(prefilter):
    r = Renderer(0)
    try:
        sc = synth.mixed_scene(5, 72, 64, scale=0.08, size_scale=0.25)
        opts = RenderOptions(samples_x=2, samples_y=2, seed=3, jitter=not prefilter, use_prefiltering=prefilter)
        pts, pp = scene_tensors(sc)
        pts.requires_grad_(True)
        pp.requires_grad_(True)
        img = render(pts, pp, r, sc, opts, BackwardOptions())
        ref_img = r.render(sc, opts).pixels
        assert float(np.max(np.abs(img.detach().cpu().numpy() - ref_img))) <= 1e-6
        w = torch.tensor(np.random.default_rng(1).normal(0, 1, ref_img.shape).astype(np.float32), device="cuda")
        (img * w).sum().backward()
        ref = r.render_backward(sc, opts, BackwardOptions(), w.cpu().numpy()).buffers
        for got, name in ((pts.grad, "d_points"), (pp.grad, "d_paint_params")):
            g = got.detach().cpu().numpy().reshape(-1)
            e = ref[name]
            scale = float(np.max(np.abs(e)))
            assert float(np.max(np.abs(g - e))) <= 1e-4 * (scale + 1e-6) + 1e-6, name
    finally:
        r.close()
