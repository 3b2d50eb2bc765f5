"""Writes profiles/roofline_work.json: the forward-pass work of the benchmark scenes
for the compute roofline, counted by brute force with the oracle's counting build.

Unit: one test the crate's BVH queries reach for one pixel sample (a path segment
whose padded bounds pass the fill ray test or contain the sample for a stroke; an
analytic shape whose bounds contain it).  Weight: the floating-point operations the
crate's arithmetic executes for that test (the winding solve, or the closest point
and the stroke radius), counted operation by operation (OPS in oracle.cpp: one per
f32 / f64 add, subtract, multiply, divide, square root and libm call).  The totals
do not depend on how a GPU kernel visits the tests or skips some of them.

Test infrastructure: bench.py only reads the JSON this writes.

    python oracle/count_work.py [--threads N]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [os.path.join(ROOT, "diffvg-rs_b200"), HERE]

import pyoracle as orc  # noqa: E402
from dvg import RenderOptions, synth  # noqa: E402

OUT = os.path.join(ROOT, "profiles", "roofline_work.json")


def workloads():
    """The bench.py workloads (same scene generators, seeds and options)."""
    large = RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=True, use_prefiltering=False)
    return {
        "mixed": (synth.mixed_scene(0), synth.mixed_options(),
                  "512x512, 4x4 spp, 256 shapes (128 cubic fills, 64 strokes, 32 circles, 32 ellipses), seed 0"),
        "plain": (synth.plain_scene(0), synth.plain_options(), "256x256, 2x2 spp, 16 closed cubic paths, seed 0"),
        "adjoint": (synth.adjoint_scene(0), synth.adjoint_options(),
                    "128x128, 4x4 spp, 4 filled cubic + 4 stroked quadratic paths, seed 0"),
        "large": (synth.large_scene(0), large, "1024x1024, 4x4 spp, 4096 closed cubic paths x 16 segments, seed 0"),
    }


def count(name: str, threads: int = 0) -> dict:
    sc, opts, label = workloads()[name]
    work = orc.count_work(sc, opts, threads)
    tests = {k: n for k, (n, _) in work.items() if n}
    return {"scene": label, "pixel_samples": sc.width * sc.height * opts.samples_x * opts.samples_y,
            "tests": tests, "flops": {k: work[k][1] for k in tests},
            "flops_per_test": {k: round(work[k][1] / n, 3) for k, n in tests.items()},
            "total_tests": sum(tests.values()), "total_flops": sum(work[k][1] for k in tests)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    out = {
        "what": "forward-pass work of the bench workloads for the compute roofline (FP32 issue): tests the crate's "
                "BVH queries reach per pixel sample and the floating-point operations of the crate's arithmetic "
                "for them; achieved = total_flops / the forward kernel's average launch time",
        "convention": "one operation per f32 or f64 add, subtract, multiply, divide, square root and libm call "
                      "(acos, cos, pow, sin, atan2); negation, comparisons, abs, min / max and conversions count "
                      "zero; per-sample work outside the tests (jitter, transforms, paint, compositing, splat) is "
                      "not counted",
        "command": "python oracle/count_work.py",
        "workloads": {name: count(name, args.threads) for name in workloads()},
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print(json.dumps({k: (v["total_tests"], v["total_flops"]) for k, v in out["workloads"].items()}))


if __name__ == "__main__":
    main()
