"""dvg_render_device_noalloc: the render entry point for callers that cannot call
cudaMalloc while rendering (its splat accumulators live in a fixed file-scope
device array).  Called through the C ABI twice in a row — the second call must
not see the first call's leftovers — and compared with dvg_render_device.
This file sorts last so that a failing run has already run every other test;
it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from dvg import Renderer, synth
from dvg.abi import RenderOptionsC, render_options_c

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same per-channel image tolerance as the other image tests


def _bind(lib):
    f = lib.dvg_render_device_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(RenderOptionsC), C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_matches_render_device_twice():
    import torch

    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    r = Renderer(0)
    noalloc = _bind(r.lib)
    for sc, opts in ((synth.mixed_scene(2), synth.mixed_options()),  # exactly the 512x512 limit
                     (synth.plain_scene(4, 200, 120, 10), synth.plain_options())):
        up = r.upload(sc)
        n = sc.width * sc.height * 4
        ref = torch.empty(n, device="cuda")
        up.render_device(opts, ref.data_ptr())
        o = render_options_c(opts)
        for _ in range(2):
            out = torch.full((n,), -1.0, device="cuda")
            st = noalloc(r.ctx, up.handle, C.byref(o), C.c_void_p(out.data_ptr()))
            assert st == 0, r.lib.dvg_last_error()
            torch.cuda.synchronize()
            err = float((out - ref).abs().max())
            assert err <= TOL, err
        up.close()
    r.close()


def test_noalloc_rejects_oversized_canvas():
    import torch

    assert torch.cuda.is_available()
    r = Renderer(0)
    noalloc = _bind(r.lib)
    up = r.upload(synth.plain_scene(0, 600, 600, 2))
    out = torch.zeros(600 * 600 * 4, device="cuda")
    o = render_options_c(synth.plain_options())
    st = noalloc(r.ctx, up.handle, C.byref(o), C.c_void_p(out.data_ptr()))
    assert st == 4  # DVG_ERR_INVALID_ARGUMENT
    assert b"no-allocation limit" in r.lib.dvg_last_error()
    assert float(out.abs().max()) == 0.0  # nothing was launched
    up.close()
    r.close()
