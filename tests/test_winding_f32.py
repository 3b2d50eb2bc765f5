"""The certified f32 decisions (diffvg-rs_b200/csrc/certified_f32.cuh, used by every
kernel before the f64 solves) against the oracle's restatement of the crate's f64
computations.  Cubic winding: random segments with query points near the curve, integer
alignments, near-degenerate cubics (elevated quadratics, lines, cusps, tiny loops),
query rows exactly at end points and extrema, large coordinates, scene-like tests.
Quadratic stroke test: query points at the stroke's edge (radius +- 10^U[-6, 1]),
nearly straight and degenerate quadratics, large coordinates, scene-like tests.  Never
a decision that differs from the f64 one; most of a scene's tests decided in f32 (so
the f64 solves run rarely)."""
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
    for fn in ("winding_stress", "within_stress"):
        getattr(L, fn).argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_float, C.POINTER(C.c_ulonglong)]
        getattr(L, fn).restype = None

    def run(fn, mode, seed, n, perturb=0.0):
        out = (C.c_ulonglong * 3)()
        getattr(L, fn)(mode, seed, n, perturb, out)
        return list(out)
    return run


# perturb: the initial roots moved by up to +-1e-3 before the refinement, twice the
# largest error of the GPU's fast root formulas (fast cos, the acos approximation, fast
# power), so the decisions hold for the device arithmetic as well as the host's.
@pytest.mark.parametrize("perturb", [0.0, 1e-3])
@pytest.mark.parametrize("mode", range(len(MODES)), ids=MODES)
def test_certified_f32_winding_never_disagrees(stress, mode, perturb):
    cases, certified, wrong = stress("winding_stress", mode, 11, 2_000_000, perturb)
    assert cases == 2_000_000
    assert wrong == 0, f"{wrong} certified decisions differ from the f64 ones ({MODES[mode]})"
    if mode == 5:
        assert certified >= 0.9 * cases, f"only {certified / cases:.3f} of a scene's tests decided in f32"


WITHIN_MODES = ("at the stroke edge", "nearly straight", "degenerate", "large coordinates", "scene tests")


@pytest.mark.parametrize("perturb", [0.0, 1e-3])
@pytest.mark.parametrize("mode", range(len(WITHIN_MODES)), ids=WITHIN_MODES)
def test_certified_f32_quadratic_stroke_never_disagrees(stress, mode, perturb):
    cases, certified, wrong = stress("within_stress", mode, 12, 2_000_000, perturb)
    assert cases == 2_000_000
    assert wrong == 0, f"{wrong} certified decisions differ from the f64 ones ({WITHIN_MODES[mode]})"
    if mode == 4:
        assert certified >= 0.9 * cases, f"only {certified / cases:.3f} of a scene's tests decided in f32"
