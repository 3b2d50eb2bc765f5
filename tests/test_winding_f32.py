"""The certified f32 cubic winding (diffvg-rs_b200/csrc/winding_f32.cuh, used by every
kernel's winding solve before the f64 one) against the oracle's restatement of the
crate's f64 computation: on random segments with query points near the curve, integer
alignments, near-degenerate cubics (elevated quadratics, lines, cusps, tiny loops),
query rows exactly at end points and extrema, large coordinates, and the tests a
scene makes, it never returns a decision that differs from the f64 one; and it
decides most of a scene's tests (so the f64 solve runs rarely)."""
import ctypes as C
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.join(os.path.dirname(HERE), "oracle")
LIB = os.path.join(ORACLE, "_build", "libwinding_stress.so")
MODES = ("near the curve", "integer alignments", "near-degenerate", "rows at end points and extrema",
         "large coordinates", "scene tests")


@pytest.fixture(scope="module")
def stress():
    subprocess.run(["make", "-s", "-C", ORACLE], check=True)
    L = C.CDLL(LIB)
    L.winding_stress.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.POINTER(C.c_ulonglong)]
    L.winding_stress.restype = None

    def run(mode, seed, n):
        out = (C.c_ulonglong * 3)()
        L.winding_stress(mode, seed, n, out)
        return list(out)
    return run


@pytest.mark.parametrize("mode", range(len(MODES)), ids=MODES)
def test_certified_f32_winding_never_disagrees(stress, mode):
    cases, certified, wrong = stress(mode, 11, 2_000_000)
    assert cases == 2_000_000
    assert wrong == 0, f"{wrong} certified decisions differ from the f64 ones ({MODES[mode]})"
    if mode == 5:
        assert certified >= 0.9 * cases, f"only {certified / cases:.3f} of a scene's tests decided in f32"
