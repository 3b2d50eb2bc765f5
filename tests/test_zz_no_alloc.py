"""dvg_render_device_noalloc: the render entry point for callers that cannot call
cudaMalloc while rendering (its splat accumulators live in a fixed file-scope
device array).  Called through the C ABI twice in a row — the second call must
not see the first call's leftovers — and compared with dvg_render_device and with
the CPU oracle, in plain and prefiltered rendering; across those calls the device's
free memory must not change (nothing is allocated).
This file sorts last so that a failing run has already run every other test;
it also passes on its own in a fresh process.
"""
import ctypes as C
import os

import numpy as np
import pytest

import pyoracle as orc
from dvg import Renderer, RenderOptions, synth
from dvg.abi import RenderOptionsC, render_options_c

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same per-channel image tolerance as the other image tests


def _bind(lib):
    f = lib.dvg_render_device_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(RenderOptionsC), C.c_void_p]
    f.restype = C.c_int
    return f


def _cases():
    prefilter = RenderOptions(samples_x=2, samples_y=2, seed=2, jitter=True, use_prefiltering=True)
    return (("mixed512", synth.mixed_scene(2), synth.mixed_options()),  # exactly the 512x512 limit
            ("plain200x120", synth.plain_scene(4, 200, 120, 10), synth.plain_options()),
            ("prefiltered", synth.plain_scene(5, 160, 144, 8), prefilter))


@pytest.mark.parametrize("name", ["mixed512", "plain200x120", "prefiltered"])
def test_noalloc_matches_render_device_and_oracle_twice(name):
    import torch

    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    sc, opts = next((s, o) for n, s, o in _cases() if n == name)
    r = Renderer(0)
    noalloc = _bind(r.lib)
    up = r.upload(sc)
    n = sc.width * sc.height * 4
    ref = torch.empty(n, device="cuda")
    up.render_device(opts, ref.data_ptr())
    o = render_options_c(opts)
    outs = [torch.full((n,), -1.0, device="cuda") for _ in range(3)]
    # first call: looks up the static array's address and loads the kernels
    st = noalloc(r.ctx, up.handle, C.byref(o), C.c_void_p(outs[0].data_ptr()))
    assert st == 0, r.lib.dvg_last_error()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for out in outs[1:]:
        st = noalloc(r.ctx, up.handle, C.byref(o), C.c_void_p(out.data_ptr()))
        assert st == 0, r.lib.dvg_last_error()
        torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before, "device memory changed across no-allocation calls"
    oracle = orc.render_window(sc, opts, 0, 0, sc.width, sc.height, threads=os.cpu_count() or 1).reshape(-1)
    for out in outs:
        assert float((out - ref).abs().max()) <= TOL
        assert float(np.max(np.abs(out.cpu().numpy().astype(np.float64) - oracle))) <= TOL
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
