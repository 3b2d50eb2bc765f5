"""The Newton-certified cubic winding (diffvg-rs_b200/csrc/winding_newton.cuh, taken by
every kernel before the crate's f64 root formula) against the oracle's restatement of
the crate's f64 computation (winding_number_segment, src/distance/winding.rs:170-192).
Random segments with query points near the curve, integer alignments, near-degenerate
cubics (elevated quadratics, lines, cusps, tiny loops), query rows exactly at end points
and extrema, large coordinates, scene-like tests and rows within 1e-12..1e-2 of a y
extremum (near double roots); the f32 root estimates also moved by up to 1e-5, 1e-4 and
8e-4 of their formula's scale 2 sqrt(q) (the device's estimates are within 1.7e-4 of it:
fast cosine, f32 acos of a rounded argument); the library skips the Newton step of a root
whose estimate lies more than 2e-3 sqrt(q) outside [0, 1], and a harness run with larger
moves (2.5e-3 of the scale) does find wrong decisions, so the cases reach that test.
Never a decision that differs from the crate's; nearly all of a scene's tests decided
without the crate's formula.

The same certified roots give the quadratic closest point's candidates (the stationarity
cubic's roots in [0, 1] as the f32 parameters the crate evaluates): against the oracle's
closest_point_quadratic (curve.rs:26-78), bit-identical point, parameter and distance on
random segments with query points near the curve, integer alignments, nearly straight and
degenerate segments, points near a centre of curvature (merging stationary points) and
scene tests."""
import ctypes as C
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.join(os.path.dirname(HERE), "oracle")
LIB = os.path.join(ORACLE, "_build", "libwinding_stress.so")
MODES = ("near the curve", "integer alignments", "near-degenerate", "rows at end points and extrema",
         "large coordinates", "scene tests", "near double roots")


@pytest.fixture(scope="module")
def stress():
    subprocess.run(["make", "-s", "-C", ORACLE], check=True)
    L = C.CDLL(LIB)
    L.winding_stress.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_float, C.POINTER(C.c_ulonglong)]
    L.winding_stress.restype = None

    def run(mode, seed, n, perturb):
        out = (C.c_ulonglong * 3)()
        L.winding_stress(mode, seed, n, perturb, out)
        return list(out)
    return run


@pytest.mark.parametrize("perturb", [0.0, 1e-5, 1e-4, 8e-4])
@pytest.mark.parametrize("mode", range(len(MODES)), ids=MODES)
def test_newton_winding_never_disagrees(stress, mode, perturb):
    cases, decided, wrong = stress(mode, 11, 2_000_000, perturb)
    assert cases == 2_000_000
    assert wrong == 0, f"{wrong} decisions differ from the crate's ({MODES[mode]})"
    if mode == 5 and perturb <= 1e-4:  # the device's estimates err by ~1e-7 of the scale, rarely more
        bar = 0.999 if perturb <= 1e-5 else 0.995
        assert decided >= bar * cases, f"only {decided / cases:.4f} of a scene's tests decided"


def test_harness_finds_wrong_decisions_beyond_the_estimate_bound(stress):
    """Estimates moved past the 2e-3 sqrt(q) skip bound: the harness must see wrong decisions."""
    wrong = sum(stress(mode, 5, 1_000_000, 2.5e-3)[2] for mode in range(len(MODES)))
    assert wrong > 0


QUAD_MODES = ("near the curve", "integer alignments", "nearly straight and degenerate", "near the evolute",
              "scene tests")


@pytest.fixture(scope="module")
def quad_stress():
    subprocess.run(["make", "-s", "-C", ORACLE], check=True)
    L = C.CDLL(LIB)
    L.closest_quad_stress.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_float, C.POINTER(C.c_ulonglong)]
    L.closest_quad_stress.restype = None

    def run(mode, seed, n, perturb):
        out = (C.c_ulonglong * 3)()
        L.closest_quad_stress(mode, seed, n, perturb, out)
        return list(out)
    return run


@pytest.mark.parametrize("perturb", [0.0, 1e-5, 1e-4])
@pytest.mark.parametrize("mode", range(len(QUAD_MODES)), ids=QUAD_MODES)
def test_newton_closest_quadratic_is_bit_identical(quad_stress, mode, perturb):
    cases, decided, wrong = quad_stress(mode, 7, 1_000_000, perturb)
    assert cases >= 900_000
    assert wrong == 0, f"{wrong} closest points differ from the crate's ({QUAD_MODES[mode]})"
    if mode == 4 and perturb == 0.0:
        assert decided >= 0.999 * cases, f"only {decided / cases:.4f} of a scene's tests decided"
