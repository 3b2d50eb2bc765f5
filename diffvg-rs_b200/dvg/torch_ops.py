"""torch.autograd bridge over the C ABI (the Python counterpart of the crate's
render / render_backward pair): path points and paint parameters are tensors, the
image is a tensor on the GPU, and backward calls dvg_render_backward_device.

Each forward prepares and uploads the scene with the tensors' current values (the
crate re-prepares on every render call too); gradients flow to `points` ([P, 2], the
scene's flattened path points in shape order) and `paint_params` ([Q, 4], one row
per group fill / stroke paint as packed by dvg.abi.pack_scene).
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .abi import pack_scene
from .renderer import DeviceGrads, Renderer
from .scene import BackwardOptions, RenderOptions, Scene


def scene_tensors(scene: Scene, device="cuda"):
    """(points [P, 2], paint_params [Q, 4]) tensors holding the scene's current values."""
    import torch

    pk = pack_scene(scene)
    pts = torch.tensor(pk.arrays["pts"].reshape(-1, 2), dtype=torch.float32, device=device)
    pp = torch.tensor(pk.arrays["p_params"].reshape(-1, 4), dtype=torch.float32, device=device)
    return pts, pp


def _render_function():
    import torch

    class RenderFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, points, paint_params, renderer: Renderer, scene: Scene, options: RenderOptions,
                    backward_options: Optional[BackwardOptions]):
            pk = pack_scene(scene)
            if points.numel() != pk.arrays["pts"].size or paint_params.numel() != pk.arrays["p_params"].size:
                raise ValueError("points / paint_params do not match the scene's layout")
            pk.arrays["pts"][:] = points.detach().float().cpu().numpy().reshape(-1)
            pk.arrays["p_params"][:] = paint_params.detach().float().cpu().numpy().reshape(-1)
            up = renderer.upload(scene, packed=pk)
            dev = torch.device("cuda", torch.cuda.current_device())
            out = torch.empty((scene.height, scene.width, 4), dtype=torch.float32, device=dev)
            lib = torch.cuda.ExternalStream(renderer.stream_handle, device=dev)
            cur = torch.cuda.current_stream(dev)
            lib.wait_stream(cur)
            up.render_device(options, out.data_ptr())
            cur.wait_stream(lib)
            ctx.up = up
            ctx.options = options
            ctx.bopts = backward_options or BackwardOptions()
            ctx.shapes = (points.shape, paint_params.shape, points.device, paint_params.device)
            ctx.lib = lib
            return out

        @staticmethod
        def backward(ctx, grad_out):
            up = ctx.up
            pshape, qshape, pdev, qdev = ctx.shapes
            dev = grad_out.device
            g = DeviceGrads(up.packed, dev, translation=ctx.bopts.compute_translation)
            d_render = grad_out.detach().float().contiguous()
            cur = torch.cuda.current_stream(dev)
            ctx.lib.wait_stream(cur)
            up.backward_device(ctx.options, ctx.bopts, d_render.data_ptr(), g)
            cur.wait_stream(ctx.lib)
            n = int(np.prod(pshape))
            m = int(np.prod(qshape))
            dp = g.tensors["d_points"][:n].reshape(pshape).to(pdev)
            dq = g.tensors["d_paint_params"][:m].reshape(qshape).to(qdev)
            up.close()
            return dp, dq, None, None, None, None

    return RenderFunction


_FN = None


def render(points, paint_params, renderer: Renderer, scene: Scene, options: Optional[RenderOptions] = None,
           backward_options: Optional[BackwardOptions] = None):
    """Differentiable render: image [H, W, 4] (un-premultiplied linear RGBA) as a
    function of `points` and `paint_params`; `scene` supplies everything else."""
    global _FN
    if _FN is None:
        _FN = _render_function()
    return _FN.apply(points, paint_params, renderer, scene, options or RenderOptions(), backward_options)
