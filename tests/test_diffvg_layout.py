"""SceneGrad.to_diffvg_layout (src/grad.rs:474-553): path gradients carry the path's
metadata and per-point buffers sized like the source path."""
import numpy as np

from dvg import BackwardOptions, RenderOptions, synth


def test_diffvg_layout_carries_path_metadata():
    import pyoracle

    sc = synth.primitives_scene()
    opts = RenderOptions(samples_x=2, samples_y=2, seed=1, use_prefiltering=False)
    img = pyoracle.render(sc, opts)
    g, _ = pyoracle.render_backward(sc, opts, BackwardOptions(), 0.1 * img)
    d = g.to_diffvg_layout(sc)
    assert len(d.shapes) == len(sc.shapes) and len(d.shape_groups) == len(sc.groups)
    for ds, sh, gs in zip(d.shapes, sc.shapes, g.shapes):
        geo = ds.geometry
        if geo["kind"] != "path":
            assert geo == gs.geometry
            continue
        path = sh.geometry.path
        assert geo["num_control_points"] == list(path.num_control_points)
        assert geo["is_closed"] == path.is_closed and geo["use_distance_approx"] == path.use_distance_approx
        assert geo["points"].shape == (len(path.points), 2)
        assert np.array_equal(geo["points"], gs.geometry["points"])
        if path.thickness is None:
            assert geo["thickness"] is None
        else:
            assert geo["thickness"].shape == (len(path.thickness),)
        assert np.array_equal(ds.transform, gs.transform) and ds.stroke_width == gs.stroke_width
    assert np.array_equal(d.background, g.background) and d.filter_radius == g.filter_radius
