"""One scene split into shards (dvg_shard_forward / _resolve / _backward): the shards
of 2 and 3 processes, run one after another on one GPU and summed as the
all-reduces would sum them, give the image (2e-6), the loss (1e-5 relative) and
the gradients (1e-4 of each array's scale: float summation order) of the
single-call fused step; a shard may hold only tiles or only boundary samples."""
import numpy as np
import pytest
import torch

from dvg import BackwardOptions, DeviceGrads, Renderer, RenderOptions, synth
from dvg.shard import shard_range

pytestmark = pytest.mark.gpu


def _full(up, opts, bo, tgt):
    n = up.scene.width * up.scene.height * 4
    out = torch.empty(n, device="cuda")
    loss = torch.zeros(1, device="cuda")
    g = DeviceGrads(up.packed, "cuda")
    torch.cuda.synchronize()
    up.fwd_bwd_l2_device(opts, bo, tgt.data_ptr(), out.data_ptr(), loss.data_ptr(), g)
    torch.cuda.synchronize()
    return out, float(loss), g


def _sharded(r, up, opts, bo, tgt, shards):
    # the library runs on its own stream, torch on the default one: synchronise between them
    npix = up.scene.width * up.scene.height
    accs = [torch.empty(npix * 5, device="cuda") for _ in shards]
    torch.cuda.synchronize()
    for (tiles, _), acc in zip(shards, accs):
        up.shard_forward(opts, tiles, acc.data_ptr(), acc.data_ptr() + npix * 16)
    torch.cuda.synchronize()
    acc = torch.stack(accs).sum(0)  # the all-reduce of the accumulators
    img = torch.empty(npix * 4, device="cuda")
    d_render = torch.empty(npix * 4, device="cuda")
    loss = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    wsum_ptr = acc.data_ptr() + npix * 16
    up.shard_resolve(acc.data_ptr(), wsum_ptr, img.data_ptr())
    r.l2_device(img.data_ptr(), tgt.data_ptr(), npix * 4, d_render.data_ptr(), loss.data_ptr())
    total = None
    for tiles, samples in shards:
        g = DeviceGrads(up.packed, "cuda")
        torch.cuda.synchronize()
        up.shard_backward(opts, bo, tiles, samples, d_render.data_ptr(), wsum_ptr, g)
        torch.cuda.synchronize()
        if total is None:
            total = g
        else:
            total.buffer += g.buffer  # the all-reduce of the gradients
    torch.cuda.synchronize()
    return img, float(loss), total


@pytest.mark.parametrize("scene", ["mixed", "styled"])
def test_shards_sum_to_the_whole_step(scene):
    r = Renderer(0)
    try:
        if scene == "mixed":
            sc = synth.mixed_scene(4, 96, 80, scale=0.1, size_scale=0.3)
        else:
            sc = synth.styled_stroke_scene(2)
        opts = RenderOptions(samples_x=2, samples_y=2, seed=3, jitter=True, use_prefiltering=False)
        nb = 5000
        bo = BackwardOptions(boundary_samples=nb)
        up = r.upload(sc)
        tgt = torch.rand(sc.width * sc.height * 4, device="cuda")
        ref_img, ref_loss, ref_g = _full(up, opts, bo, tgt)
        tiles = up.tile_count()
        cases = [[(shard_range(tiles, k, w), shard_range(nb, k, w)) for k in range(w)] for w in (2, 3)]
        cases.append([((0, tiles), (0, 0)), ((tiles, tiles), (0, nb))])  # tiles only, samples only
        for shards in cases:
            img, loss, g = _sharded(r, up, opts, bo, tgt, shards)
            assert float(torch.max(torch.abs(img - ref_img))) <= 2e-6, shards
            assert abs(loss - ref_loss) <= 1e-5 * abs(ref_loss) + 1e-6, shards
            for k, v in ref_g.tensors.items():
                a, b = g.tensors[k].cpu().numpy(), v.cpu().numpy()
                scale = float(np.max(np.abs(b))) if b.size else 0.0
                assert float(np.max(np.abs(a - b))) <= 1e-4 * (scale + 1e-6) + 1e-6, (shards, k)
        up.close()
    finally:
        r.close()


def test_tuning_change_between_shard_calls():
    """dvg_scene_set_tuning between dvg_shard_forward and dvg_shard_backward: the
    forward's fragment codes were laid out for the old slot count and sample layout,
    so the backward must rebuild the fragments instead of reading them; its
    gradients equal a fresh fused step under the new tuning."""
    r = Renderer(0)
    try:
        sc = synth.mixed_scene(4, 96, 80, scale=0.1, size_scale=0.3)
        opts = RenderOptions(samples_x=2, samples_y=2, seed=3, jitter=True, use_prefiltering=False)
        nb = 5000
        bo = BackwardOptions(boundary_samples=nb)
        up = r.upload(sc)
        tgt = torch.rand(sc.width * sc.height * 4, device="cuda")
        tiles = up.tile_count()
        npix = sc.width * sc.height
        for before, after in (((1, 4, 8), (1, 4, 32)), ((1, 4, 16), (0, 4, 16)), ((0, 2, 32), (1, 8, 0))):
            up.set_tuning(*after)
            ref_img, _, ref_g = _full(up, opts, bo, tgt)
            up.set_tuning(*before)
            acc = torch.empty(npix * 5, device="cuda")
            torch.cuda.synchronize()
            up.shard_forward(opts, (0, tiles), acc.data_ptr(), acc.data_ptr() + npix * 16)
            img = torch.empty(npix * 4, device="cuda")
            d_render = torch.empty(npix * 4, device="cuda")
            up.shard_resolve(acc.data_ptr(), acc.data_ptr() + npix * 16, img.data_ptr())
            r.l2_device(img.data_ptr(), tgt.data_ptr(), npix * 4, d_render.data_ptr(), 0)
            up.set_tuning(*after)
            g = DeviceGrads(up.packed, "cuda")
            torch.cuda.synchronize()
            up.shard_backward(opts, bo, (0, tiles), (0, nb), d_render.data_ptr(), acc.data_ptr() + npix * 16, g)
            torch.cuda.synchronize()
            assert float(torch.max(torch.abs(img - ref_img))) <= 2e-6
            for k, v in ref_g.tensors.items():
                a, b = g.tensors[k].cpu().numpy(), v.cpu().numpy()
                scale = float(np.max(np.abs(b))) if b.size else 0.0
                assert float(np.max(np.abs(a - b))) <= 1e-4 * (scale + 1e-6) + 1e-6, (before, after, k)
        up.close()
    finally:
        r.close()


def test_shard_ranges_are_checked():
    from dvg.renderer import RenderError

    r = Renderer(0)
    try:
        up = r.upload(synth.plain_scene(1, 64, 48, 4))
        tiles = up.tile_count()
        assert tiles == 4 * 3
        acc = torch.empty(64 * 48 * 5, device="cuda")
        torch.cuda.synchronize()
        opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=True, use_prefiltering=False)
        with pytest.raises(RenderError):
            up.shard_forward(opts, (0, tiles + 1), acc.data_ptr(), acc.data_ptr() + 64 * 48 * 16)
        with pytest.raises(RenderError):
            up.shard_forward(opts, (3, 2), acc.data_ptr(), acc.data_ptr() + 64 * 48 * 16)
        up.close()
    finally:
        r.close()
