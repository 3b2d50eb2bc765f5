"""Launch-shape tuning (dvg_tuning): every warp layout, boundary cell and
fragment-cache size gives the same image (to float-atomic order, 2e-6) and
gradients (1e-4 of scale) as the default; the autotuners pick a valid shape, for a
scene and for a batch.  Cache sizes of 1 and 2 slots leave many samples over the
cap, so warps mix cached samples with samples that repeat the hit tests."""
import numpy as np
import pytest
import torch

from dvg import BackwardOptions, Batch, DeviceGrads, Renderer, RenderOptions, synth

pytestmark = pytest.mark.gpu

# (sample_layout, boundary_cell, fragment_slots[, work_queue, forward_occupancy])
SHAPES = [(1, 4, 16), (0, 4, 16), (1, 2, 16), (1, 8, 16), (1, 16, 16), (0, 16, 16), (1, 4, 0), (0, 4, 0),
          (1, 4, 1), (0, 4, 2), (1, 4, 8), (1, 4, 64), (1, 4, 16, 0, 1), (0, 2, 0, 0, 1), (1, 4, 16, 0, 2)]


def _run(up, opts, bo, tgt):
    n = up.scene.width * up.scene.height * 4
    out = torch.empty(n, device="cuda")
    loss = torch.zeros(1, device="cuda")
    g = DeviceGrads(up.packed, "cuda")
    torch.cuda.synchronize()
    up.fwd_bwd_l2_device(opts, bo, tgt.data_ptr(), out.data_ptr(), loss.data_ptr(), g)
    torch.cuda.synchronize()
    return out.cpu().numpy(), {k: v.cpu().numpy() for k, v in g.tensors.items()}


@pytest.mark.parametrize("prefilter", [False, True])
def test_every_launch_shape_gives_the_same_result(prefilter):
    r = Renderer(0)
    try:
        sc = synth.mixed_scene(11, 96, 80, scale=0.1, size_scale=0.3)
        opts = RenderOptions(samples_x=3, samples_y=2, seed=2, jitter=not prefilter, use_prefiltering=prefilter)
        bo = BackwardOptions(boundary_samples=4000)
        up = r.upload(sc)
        t = r.upload(synth.plain_scene(5, 96, 80, 6))
        tgt = torch.empty(96 * 80 * 4, device="cuda")
        t.render_device(opts, tgt.data_ptr())
        ref_img, ref_g = _run(up, opts, bo, tgt)
        for shape in SHAPES:
            up.set_tuning(*shape)
            assert up.tuning()[:len(shape)] == tuple(shape)
            img, g = _run(up, opts, bo, tgt)
            assert float(np.max(np.abs(img - ref_img))) <= 2e-6, shape
            for k, v in ref_g.items():
                scale = float(np.max(np.abs(v))) if v.size else 0.0
                assert float(np.max(np.abs(g[k] - v))) <= 1e-4 * (scale + 1e-6) + 1e-6, (shape, k)
        chosen = up.autotune(opts, bo, tgt.data_ptr())
        assert chosen[0] in (0, 1) and chosen[1] in (2, 4, 8, 16) and chosen[2] <= 64 and up.tuning() == chosen
        img, _ = _run(up, opts, bo, tgt)
        assert float(np.max(np.abs(img - ref_img))) <= 2e-6
        t.close()
        up.close()
    finally:
        r.close()


def _batch_grads(batch, i, ups):
    import ctypes as C

    from dvg import device_view

    _, _, g = batch.buffers(i)
    d = ups[i].packed.desc
    pts = device_view(C.cast(g.d_points, C.c_void_p).value, 2 * d.total_points).cpu().numpy()
    pp = device_view(C.cast(g.d_paint_params, C.c_void_p).value, 4 * d.num_paints).cpu().numpy()
    return pts, pp


def test_batch_autotune_keeps_results():
    r = Renderer(0)
    try:
        scenes = [synth.plain_scene(30 + i, 48 + 16 * i, 40, 4 + i) for i in range(3)]
        opts = RenderOptions(samples_x=2, samples_y=2, seed=1, jitter=True, use_prefiltering=False)
        ups = [r.upload(s) for s in scenes]
        b = Batch(r, ups, opts, BackwardOptions(boundary_samples=1500))
        for i, s in enumerate(scenes):
            t = r.upload(synth.plain_scene(50 + i, s.width, s.height, 5))
            _, tgt, _ = b.buffers(i)
            t.render_device(opts, tgt.data_ptr())
            torch.cuda.synchronize()
            t.close()
        b.step(False)
        ref = b.losses().copy()
        chosen = b.autotune()
        assert chosen[0] in (0, 1) and chosen[1] in (2, 4, 8, 16) and chosen[2] in (0, 8, 16, 32)
        assert chosen[3] in (0, 1) and chosen[4] in (0, 1, 2)
        b.step(True)
        assert np.allclose(b.losses(), ref, rtol=1e-5, atol=1e-6)
        # gradients with and without the fragment cache, one CTA per work item or persistent CTAs,
        # the forward at 2 or 3 CTAs per SM
        grads = []
        for slots, queue, occ in ((0, 0, 0), (2, 0, 0), (16, 0, 0), (16, 1, 0), (0, 1, 0), (16, 0, 1), (16, 1, 1), (16, 0, 2)):
            b.set_tuning(1, 4, slots, queue, occ)
            b.step(True)
            b.losses()
            grads.append([(lambda g: (g[0].copy(), g[1].copy()))(_batch_grads(b, i, ups)) for i in range(3)])
        for other in grads[1:]:
            for (p0, c0), (p1, c1) in zip(grads[0], other):
                for x, y in ((p1, p0), (c1, c0)):
                    scale = float(np.max(np.abs(y))) if y.size else 0.0
                    assert float(np.max(np.abs(x - y))) <= 1e-4 * (scale + 1e-6) + 1e-6
        b.close()
        for u in ups:
            u.close()
    finally:
        r.close()
