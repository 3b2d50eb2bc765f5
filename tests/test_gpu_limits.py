"""Bounded device loops report instead of truncating: a sample covered by more
fragments than the interior adjoint's per-thread capacity (96; 48 prefiltered)
makes render_backward fail with DVG_ERR_DEVICE_LIMIT, the forward still renders,
and the context stays usable for the next call."""
import numpy as np
import pytest

from dvg import BackwardOptions, Color, Rect, RenderOptions, Renderer, Scene, Shape, ShapeGroup, synth
from dvg.renderer import RenderError

pytestmark = pytest.mark.gpu

DVG_ERR_DEVICE_LIMIT = 3


def _deep_scene(layers):
    sc = Scene(32, 32)
    sc.background = Color(1, 1, 1, 1)
    for i in range(layers):
        sc.shapes.append(Shape(Rect((1.0 + 0.01 * i, 1.0), (31.0, 31.0))))
        sc.groups.append(ShapeGroup([i], Color(0.5, 0.01 * i, 0.2, 0.05), None))
    return sc


@pytest.mark.parametrize("prefilter,layers", [(False, 100), (True, 60)])
def test_fragment_overflow_is_reported(prefilter, layers):
    r = Renderer(0)
    try:
        sc = _deep_scene(layers)
        opts = RenderOptions(samples_x=1, samples_y=1, seed=0, jitter=False, use_prefiltering=prefilter)
        img = r.render(sc, opts).pixels
        assert np.all(np.isfinite(img))
        with pytest.raises(RenderError) as ei:
            r.render_backward(sc, opts, BackwardOptions(), np.ones((32, 32, 4), np.float32))
        assert ei.value.status == DVG_ERR_DEVICE_LIMIT
        ok = synth.plain_scene(0, 32, 32, 3)  # the context still works afterwards
        g = r.render_backward(ok, opts, BackwardOptions(), np.ones((32, 32, 4), np.float32))
        assert np.all(np.isfinite(g.buffers["d_paint_params"]))
    finally:
        r.close()
