"""Regenerates tests/golden/golden.npz from the CPU oracle.

    python tests/golden/make_golden.py

Each render case stores the image; each backward case stores the oracle image,
the seeded d_render it is differentiated against, and every gradient array.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "diffvg-rs_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import pyoracle  # noqa: E402
from cases import CASES, build, d_render_for  # noqa: E402


def main():
    out = {}
    for name in CASES:
        sc, opts, bopts = build(name)
        img = pyoracle.render(sc, opts)
        out[f"{name}.image"] = img
        if bopts is not None:
            dr = d_render_for(img)
            _, buf = pyoracle.render_backward(sc, opts, bopts, dr, threads=1)
            out[f"{name}.d_render"] = dr
            for n in buf.NAMES:
                if buf[n] is not None:
                    out[f"{name}.{n}"] = np.asarray(buf[n], np.float32)
        print(name, "ok")
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)


if __name__ == "__main__":
    main()
