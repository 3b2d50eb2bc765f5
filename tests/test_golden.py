"""Committed golden fixtures (tests/golden/golden.npz, written by
tests/golden/make_golden.py from the oracle).

CPU: the oracle still reproduces every fixture (guards the checker itself).
GPU: the CUDA path through the C ABI matches every fixture — images within
1e-5 absolute per channel, gradients within 1e-4 relative (atol 1e-6) — with the
fixture's stored d_render as the adjoint input.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import CASES, build  # noqa: E402

IMG_TOL = 1e-5
GRAD_RTOL = 1e-4


@pytest.fixture(scope="module")
def golden():
    with np.load(os.path.join(HERE, "golden", "golden.npz")) as z:
        return {k: z[k] for k in z.files}


def _grad_names(golden, name):
    pre = name + "."
    return [k[len(pre):] for k in golden if k.startswith(pre) and k[len(pre):] not in ("image", "d_render")]


def _check_grads(got, golden, name, rtol):
    for n in _grad_names(golden, name):
        ref = golden[f"{name}.{n}"]
        g = np.asarray(got[n], np.float32)
        scale = float(np.max(np.abs(ref))) if ref.size else 0.0
        err = float(np.max(np.abs(g - ref))) if ref.size else 0.0
        assert err <= rtol * (scale + 1e-6) + 1e-6, f"{name}.{n}: err {err:.3e} scale {scale:.3e}"


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(golden, name):
    import pyoracle

    sc, opts, bopts = build(name)
    img = pyoracle.render(sc, opts)
    assert float(np.max(np.abs(img - golden[f"{name}.image"]))) <= 1e-6
    if bopts is not None:
        _, buf = pyoracle.render_backward(sc, opts, bopts, golden[f"{name}.d_render"], threads=1)
        _check_grads(buf, golden, name, 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_cuda_matches_golden(golden, name):
    from dvg import Renderer

    sc, opts, bopts = build(name)
    r = Renderer(0)
    try:
        img = r.render(sc, opts).pixels
        assert float(np.max(np.abs(img - golden[f"{name}.image"]))) <= IMG_TOL
        if bopts is not None:
            g = r.render_backward(sc, opts, bopts, golden[f"{name}.d_render"])
            _check_grads(g.buffers, golden, name, GRAD_RTOL)
    finally:
        r.close()
