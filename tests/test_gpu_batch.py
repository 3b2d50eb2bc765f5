"""Batched stepping (dvg_batch_*): every scene of a batch — uneven canvases and
shape counts — gets the same image, loss and gradients as a single-scene
dvg_fwd_bwd_l2_device call, both when the step is enqueued directly and when it
is replayed from its CUDA graph."""
import ctypes as C

import numpy as np
import pytest

from dvg import BackwardOptions, Batch, DeviceGrads, Renderer, RenderOptions, device_view, synth
from dvg.abi import GradBuffers

pytestmark = pytest.mark.gpu


def _scenes():
    return [synth.plain_scene(10, 64, 48, 5), synth.plain_scene(11, 128, 128, 20),
            synth.mixed_scene(12, 96, 80, scale=0.1, size_scale=0.3), synth.plain_scene(13, 32, 32, 3)]


def _grad_tensors(gc, packed):
    d = packed.desc
    sizes = dict(d_shape_params=4 * d.num_shapes, d_shape_transform=9 * d.num_shapes,
                 d_shape_stroke_width=d.num_shapes, d_points=2 * d.total_points, d_thickness=d.total_points,
                 d_group_transform=9 * d.num_groups, d_paint_params=4 * d.num_paints, d_stop_offsets=d.total_stops,
                 d_stop_colors=4 * d.total_stops, d_filter_radius=1, d_background=4)
    out = {}
    for n, sz in sizes.items():
        if sz:
            out[n] = device_view(C.cast(getattr(gc, n), C.c_void_p).value, sz).cpu().numpy()
    return out


@pytest.mark.parametrize("prefilter", [False, True])
def test_batch_matches_single_scene(prefilter):
    import torch

    r = Renderer(0)
    opts = RenderOptions(samples_x=2, samples_y=2, seed=3, jitter=True, use_prefiltering=prefilter)
    bopts = BackwardOptions()
    scenes = _scenes()
    ups = [r.upload(s) for s in scenes]
    targets = [r.upload(synth.plain_scene(100 + i, s.width, s.height, 4)) for i, s in enumerate(scenes)]
    batch = Batch(r, ups, opts, bopts)
    refs = []
    for i, (up, tu) in enumerate(zip(ups, targets)):
        img_b, tgt_b, _ = batch.buffers(i)
        tu.render_device(opts, tgt_b.data_ptr())
        n = up.scene.width * up.scene.height * 4
        out = torch.empty(n, device="cuda")
        loss = torch.zeros(1, device="cuda")
        g = DeviceGrads(up.packed, "cuda")
        up.fwd_bwd_l2_device(opts, bopts, tgt_b.data_ptr(), out.data_ptr(), loss.data_ptr(), g)
        torch.cuda.synchronize()
        refs.append((out.cpu().numpy(), float(loss.item()), {k: v.cpu().numpy() for k, v in g.tensors.items()}))
    for use_graph in (False, True, True):
        batch.step(use_graph)
        losses = batch.losses()
        for i, up in enumerate(ups):
            img_b, _, gc = batch.buffers(i)
            ref_img, ref_loss, ref_g = refs[i]
            assert float(np.max(np.abs(img_b.cpu().numpy() - ref_img))) <= 1e-5
            assert abs(losses[i] - ref_loss) <= 1e-4 * abs(ref_loss) + 1e-5
            got = _grad_tensors(gc, up.packed)
            for name, val in got.items():
                ref = ref_g[name][: val.size]
                scale = float(np.max(np.abs(ref))) + 1e-6
                assert float(np.max(np.abs(val - ref))) <= 1e-4 * scale + 1e-6, (i, name, use_graph)
    batch.close()
    r.close()
