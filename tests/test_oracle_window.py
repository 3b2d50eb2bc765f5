"""The oracle's windowed, threaded render (the CPU side of the configured-size
parity tests) equals the serial full-image render bit for bit on every window."""
import numpy as np
import pytest

import pyoracle as orc
from dvg import RenderOptions, synth


@pytest.mark.parametrize("case", ["plain", "mixed", "radius2", "prefilter"])
def test_window_equals_full_render(case):
    if case == "plain":
        sc, opts = synth.plain_scene(3, 72, 56, 6), synth.plain_options()
    elif case == "mixed":
        sc, opts = synth.mixed_scene(5, 64, 64, scale=0.06, size_scale=0.2), synth.mixed_options()
    elif case == "radius2":
        sc = synth.plain_scene(4, 48, 40, 5)
        sc.filter.filter_type, sc.filter.radius = 1, 2.0  # tent, two pixels of reach
        opts = RenderOptions(samples_x=3, samples_y=2, seed=9, jitter=True, use_prefiltering=False)
    else:
        sc = synth.plain_scene(6, 40, 40, 4)
        opts = RenderOptions(samples_x=2, samples_y=2, seed=1, jitter=False, use_prefiltering=True)
    full = orc.render(sc, opts)
    H, W = full.shape[:2]
    for x0, y0, x1, y1 in ((0, 0, W, H), (0, 16, W, 32), (5, 3, 29, 17), (W - 7, H - 5, W, H)):
        win = orc.render_window(sc, opts, x0, y0, x1, y1, threads=4)
        assert win.shape == (y1 - y0, x1 - x0, 4)
        assert np.array_equal(win, full[y0:y1, x0:x1]), (case, x0, y0, x1, y1)
