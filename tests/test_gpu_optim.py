"""On-device optimisation step of a batch (dvg_batch_set_adam).

1. One step's Adam update equals a numpy restatement of PyTorch's Adam applied to
   the gradients that step produced (rel 1e-6).
2. After several graph-replayed steps the re-prepared scene tables equal a fresh
   upload of the updated scene byte for byte (dvg_scene_digest over every table,
   the tile offsets and entries), and the image of the batch's scene handle matches the
   fresh scene's image to float-atomic order (tile halos are splatted by
   neighbouring CTAs; 2e-6 absolute), and its gradients match within the parity
   bar — with and without prefiltering (prefiltered
   gradients depend on the BVH leaf order through closest-point ties).
3. Fitting a seeded target lowers the loss.
"""
import numpy as np
import pytest
import torch

from dvg import BackwardOptions, Batch, DeviceGrads, Renderer, RenderOptions, synth
from dvg.abi import scene_with_params

pytestmark = pytest.mark.gpu

LR, B1, B2, EPS = 0.05, 0.9, 0.999, 1e-8


def _scenes():
    return [synth.plain_scene(20, 64, 48, 5), synth.mixed_scene(21, 96, 80, scale=0.1, size_scale=0.3),
            synth.primitives_scene(), synth.plain_scene(23, 128, 128, 24)]


def _setup(r, opts, scenes=None):
    scenes = scenes or _scenes()
    ups = [r.upload(s) for s in scenes]
    batch = Batch(r, ups, opts, BackwardOptions(boundary_samples=2000))
    for i, s in enumerate(scenes):
        t = r.upload(synth.plain_scene(100 + i, s.width, s.height, 6))
        _, tgt, _ = batch.buffers(i)
        t.render_device(opts, tgt.data_ptr())
        torch.cuda.synchronize()
        t.close()
    return scenes, ups, batch


def _grads(batch, i, ups):
    import ctypes as C

    from dvg import device_view

    _, _, g = batch.buffers(i)
    d = ups[i].packed.desc
    pts = device_view(C.cast(g.d_points, C.c_void_p).value, 2 * d.total_points).cpu().numpy() \
        if d.total_points else np.zeros(0, np.float32)
    pp = device_view(C.cast(g.d_paint_params, C.c_void_p).value, 4 * d.num_paints).cpu().numpy()
    return pts, pp


def _adam_ref(p, g):
    g = g.astype(np.float32)
    m = np.float32(1 - B1) * g
    v = np.float32(1 - B2) * (g * g)
    bc1, bc2 = np.float32(1 - B1), np.float32(1 - B2)
    denom = np.sqrt(v) / np.sqrt(bc2) + np.float32(EPS)
    return (p - (np.float32(LR) / bc1) * (m / denom)).astype(np.float32)


def test_adam_step_matches_reference():
    r = Renderer(0)
    try:
        opts = RenderOptions(samples_x=2, samples_y=2, seed=1, jitter=True, use_prefiltering=False)
        scenes, ups, batch = _setup(r, opts)
        p0 = [(u.packed.arrays["pts"].copy(), u.packed.arrays["p_params"].copy()) for u in ups]
        batch.set_adam(LR, (B1, B2), EPS, points=True, paints=True)
        batch.step(False)
        batch.losses()  # synchronises the context stream
        for i in range(len(scenes)):
            g_pts, g_pp = _grads(batch, i, ups)
            pts, pp = batch.scene_params(i)
            ref_pts = _adam_ref(p0[i][0], g_pts).reshape(-1, 2)
            ref_pp = _adam_ref(p0[i][1], g_pp).reshape(-1, 4)
            assert np.allclose(pts, ref_pts, rtol=1e-6, atol=1e-6), i
            assert np.allclose(pp, ref_pp, rtol=1e-6, atol=1e-6), i
        batch.close()
        for u in ups:
            u.close()
    finally:
        r.close()


@pytest.mark.parametrize("prefilter", [False, True])
def test_reprepared_scene_equals_fresh_upload(prefilter):
    r = Renderer(0)
    try:
        opts = RenderOptions(samples_x=2, samples_y=2, seed=3, jitter=not prefilter, use_prefiltering=prefilter)
        scenes, ups, batch = _setup(r, opts)
        batch.set_adam(LR, (B1, B2), EPS, points=True, paints=False)
        for _ in range(4):
            batch.step(True)
        batch.losses()
        for i, sc in enumerate(scenes):
            pts, _ = batch.scene_params(i)
            assert np.all(np.isfinite(pts))
            moved = float(np.max(np.abs(pts.reshape(-1) - ups[i].packed.arrays["pts"]))) if pts.size else 1.0
            assert moved > 1e-3, i
            fresh = r.upload(scene_with_params(sc, ups[i].packed, pts))
            assert ups[i].digest() == fresh.digest(), f"scene {i}: re-prepared tables differ from a fresh upload"
            n = sc.width * sc.height * 4
            a = torch.empty(n, device="cuda")
            b = torch.empty(n, device="cuda")
            ups[i].render_device(opts, a.data_ptr())
            fresh.render_device(opts, b.data_ptr())
            torch.cuda.synchronize()
            diff = float(torch.max(torch.abs(a - b)))
            assert diff <= 2e-6, f"scene {i}: re-prepared image differs from a fresh upload by {diff:.3e}"
            tgt = torch.rand(n, device="cuda")
            out_a, out_b = torch.empty(n, device="cuda"), torch.empty(n, device="cuda")
            la, lb = torch.zeros(1, device="cuda"), torch.zeros(1, device="cuda")
            ga, gb = DeviceGrads(ups[i].packed, "cuda"), DeviceGrads(fresh.packed, "cuda")
            bo = BackwardOptions(boundary_samples=3000)
            torch.cuda.synchronize()
            ups[i].fwd_bwd_l2_device(opts, bo, tgt.data_ptr(), out_a.data_ptr(), la.data_ptr(), ga)
            fresh.fwd_bwd_l2_device(opts, bo, tgt.data_ptr(), out_b.data_ptr(), lb.data_ptr(), gb)
            torch.cuda.synchronize()
            for name in ("d_points", "d_paint_params", "d_shape_stroke_width", "d_background"):
                x, y = ga.tensors[name].cpu().numpy(), gb.tensors[name].cpu().numpy()
                if y.size == 0:
                    continue
                scale = float(np.max(np.abs(y)))
                assert float(np.max(np.abs(x - y))) <= 1e-4 * (scale + 1e-6) + 1e-6, (i, name)
            fresh.close()
        batch.close()
        for u in ups:
            u.close()
    finally:
        r.close()


def test_fitting_lowers_the_loss():
    r = Renderer(0)
    try:
        opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=True, use_prefiltering=False)
        scenes = [synth.plain_scene(40 + i, 64, 64, 6) for i in range(3)]
        _, ups, batch = _setup(r, opts, scenes)
        batch.set_adam(0.5, (B1, B2), EPS, points=True, paints=True)
        batch.step(True)
        first = batch.losses().copy()
        for _ in range(30):
            batch.step(True)
        last = batch.losses()
        assert np.all(last < first), (first, last)
        batch.close()
        for u in ups:
            u.close()
    finally:
        r.close()
