"""GPU parity at the benchmark configurations' full sizes, against the CPU oracle.

* plain     256x256, 2x2 spp, box r=0.5, 16 closed cubic paths: image, then the
            gradients of the L2 loss against the seed-1 scene's render (the
            crate's default W*H*spp PCG32 boundary samples).
* mixed     512x512, 4x4 spp, Gaussian r=1, 256 shapes: image, and the gradients
            with W*H PCG32 boundary samples.
* mixed, the crate's default options (prefiltered, 2x2 spp): image and gradients.
* adjoint   128x128, 4x4 spp, 8 paths, through the fused device call with the
            fragment cache off (fragment_slots = 0: every fragment list is rebuilt
            from the BVHs, nothing stored between the passes).
* large     1024x1024, 4x4 spp, 4096 closed cubic paths x 16 segments: two bands
            of 16x16 tiles through dvg_shard_forward + dvg_shard_resolve against
            the oracle's render of the same pixels.

Bars (the same as tests/test_gpu_parity.py): images max |gpu - oracle| <= 1e-5 per
channel; gradients, per array, max |gpu - oracle| <= 1e-4 * (max |oracle| + 1e-6)
+ 1e-6 (the boundary samples are the same PCG32 draws on both sides, so only the
float summation order of the atomics differs).  The oracle runs on every host core.
"""
import os

import numpy as np
import pytest
import torch

import pyoracle as orc
from dvg import BackwardOptions, DeviceGrads, Renderer, RenderOptions, synth

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
GRAD_RTOL = 1e-4
THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def renderer():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    r = Renderer(0)
    yield r
    r.close()


def _img_err(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))


def _grad_check(get, ref):
    for n in ref.NAMES:
        g, r = get(n), ref[n]
        if g is None or r is None:
            continue
        scale = float(np.max(np.abs(r))) if r.size else 0.0
        err = float(np.max(np.abs(g[: r.size] - r))) if r.size else 0.0
        assert err <= GRAD_RTOL * (scale + 1e-6) + 1e-6, f"{n}: max err {err:.3e} vs scale {scale:.3e}"


def _full_oracle_image(sc, opts):
    return orc.render_window(sc, opts, 0, 0, sc.width, sc.height, threads=THREADS)


def _image_and_grads(renderer, sc, target_sc, opts, bopts):
    """dvg_render + dvg_render_backward (host calls) against the oracle, d_render from
    the GPU image so both sides differentiate the same loss gradient."""
    img = renderer.render(sc, opts).pixels
    ref = _full_oracle_image(sc, opts)
    assert _img_err(img, ref) <= IMG_TOL
    target = _full_oracle_image(target_sc, opts)
    d_render = (2.0 * (img - target)).astype(np.float32)
    g = renderer.render_backward(sc, opts, bopts, d_render)
    _, rb = orc.render_backward(sc, opts, bopts, d_render, threads=THREADS)
    _grad_check(lambda n: g.buffers[n], rb)


def test_plain_256_full_size(renderer):
    _image_and_grads(renderer, synth.plain_scene(0), synth.plain_scene(1), synth.plain_options(), BackwardOptions())


def test_mixed_512_full_size(renderer):
    sc = synth.mixed_scene(0)
    _image_and_grads(renderer, sc, synth.mixed_scene(1), synth.mixed_options(),
                     BackwardOptions(boundary_samples=sc.width * sc.height))


def test_mixed_512_crate_default_options(renderer):
    """The crate's default RenderOptions (prefiltered coverage, 2x2 spp, jitter, seed 0) on
    the mixed scene: the prefiltered forward (its own translation unit, the crate's root
    formulas) and the prefiltered interior adjoint (no boundary pass in this mode)."""
    sc = synth.mixed_scene(0)
    _image_and_grads(renderer, sc, synth.mixed_scene(1), RenderOptions(), BackwardOptions())


def test_adjoint_128_recompute_path(renderer):
    sc, opts = synth.adjoint_scene(0), synth.adjoint_options()
    bopts = BackwardOptions()
    up = renderer.upload(sc)
    up.set_tuning(1, 4, 0)  # fragment cache off: the interior adjoint rebuilds every fragment list
    target = _full_oracle_image(synth.adjoint_scene(1), opts)
    n = sc.width * sc.height * 4
    tgt = torch.from_numpy(target.reshape(-1).copy()).cuda()
    out = torch.empty(n, device="cuda")
    loss = torch.zeros(1, device="cuda")
    g = DeviceGrads(up.packed, "cuda")
    torch.cuda.synchronize()
    up.fwd_bwd_l2_device(opts, bopts, tgt.data_ptr(), out.data_ptr(), loss.data_ptr(), g)
    torch.cuda.synchronize()
    img = out.cpu().numpy().reshape(sc.height, sc.width, 4)
    assert _img_err(img, _full_oracle_image(sc, opts)) <= IMG_TOL
    d_render = (2.0 * (img - target)).astype(np.float32)
    ref_loss = float(np.sum((img.astype(np.float64) - target) ** 2))
    assert abs(float(loss) - ref_loss) <= 1e-5 * ref_loss + 1e-6
    _, rb = orc.render_backward(sc, opts, bopts, d_render, threads=THREADS)
    _grad_check(lambda k: g.tensors[k].cpu().numpy() if k in g.tensors else None, rb)
    up.close()


@pytest.mark.parametrize("tile_rows", [(0, 2), (31, 33)])
def test_large_1024_tile_bands(renderer, tile_rows):
    sc = synth.large_scene(0)
    opts = RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=True, use_prefiltering=False)
    up = renderer.upload(sc)
    tiles_x = (sc.width + 15) // 16
    t0, t1 = tile_rows[0] * tiles_x, tile_rows[1] * tiles_x
    npix = sc.width * sc.height
    acc = torch.empty(npix * 5, device="cuda")
    img = torch.empty(npix * 4, device="cuda")
    torch.cuda.synchronize()
    up.shard_forward(opts, (t0, t1), acc.data_ptr(), acc.data_ptr() + npix * 16)
    up.shard_resolve(acc.data_ptr(), acc.data_ptr() + npix * 16, img.data_ptr())
    torch.cuda.synchronize()
    gpu = img.cpu().numpy().reshape(sc.height, sc.width, 4)
    # rows whose whole filter footprint lies inside the band (complete sums on the GPU side)
    ri = int(np.ceil(sc.filter.radius))
    y0 = tile_rows[0] * 16 + (ri if tile_rows[0] > 0 else 0)
    y1 = tile_rows[1] * 16 - (ri if tile_rows[1] * 16 < sc.height else 0)
    ref = orc.render_window(sc, opts, 0, y0, sc.width, y1, threads=THREADS)
    assert _img_err(gpu[y0:y1], ref) <= IMG_TOL
    up.close()
