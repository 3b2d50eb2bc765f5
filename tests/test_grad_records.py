"""Host-side gradient records: SceneGrad's per-shape and per-group entries are built on
first read from the flat buffers (src/grad.rs:113-126 layout), and read the same
values an eager copy would."""
import numpy as np
import pytest

from dvg import synth
from dvg.abi import PAINT_LINEAR, PAINT_SOLID, GradBuffers, LazyList, pack_scene, unflatten_grads
from dvg.scene import Circle, Ellipse, Rect


def _filled(packed, seed=0):
    buf = GradBuffers(packed)
    rng = np.random.default_rng(seed)
    for n in buf.NAMES:
        if buf[n] is not None:
            buf[n][:] = rng.standard_normal(buf[n].size).astype(np.float32)
    return buf


def test_records_match_flat_buffers():
    sc = synth.mixed_scene(0, 128, 128)
    p = pack_scene(sc)
    buf = _filled(p)
    g = unflatten_grads(sc, p, buf)
    assert len(g.shapes) == len(sc.shapes) and len(g.shape_groups) == len(sc.groups)
    for i, sh in enumerate(sc.shapes):
        ds = g.shapes[i]
        np.testing.assert_array_equal(ds.transform.reshape(-1), buf["d_shape_transform"][9 * i: 9 * i + 9])
        assert ds.stroke_width == float(buf["d_shape_stroke_width"][i])
        sp = buf["d_shape_params"][4 * i: 4 * i + 4]
        geo = sh.geometry
        if isinstance(geo, Circle):
            assert ds.geometry["kind"] == "circle" and ds.geometry["radius"] == float(sp[2])
        elif isinstance(geo, Ellipse):
            assert ds.geometry["kind"] == "ellipse"
            np.testing.assert_array_equal(ds.geometry["radius"], sp[2:])
        elif isinstance(geo, Rect):
            assert ds.geometry["kind"] == "rect"
        else:
            o, n = p.path_point_offset[i], p.path_point_count[i]
            np.testing.assert_array_equal(ds.geometry["points"].reshape(-1), buf["d_points"][2 * o: 2 * (o + n)])
            assert (ds.geometry["thickness"] is None) == (geo.path.thickness is None)
    for gi, grp in enumerate(sc.groups):
        dg = g.shape_groups[gi]
        np.testing.assert_array_equal(dg.shape_to_canvas.reshape(-1), buf["d_group_transform"][9 * gi: 9 * gi + 9])
        for which in ("fill", "stroke"):
            paint, rec = getattr(grp, which), getattr(dg, which)
            assert (paint is None) == (rec is None)
            if rec is None:
                continue
            pi = p.paint_of[(gi, which)]
            kind = int(p.arrays["p_kind"][pi])
            assert rec["kind"] == {PAINT_SOLID: "solid", PAINT_LINEAR: "linear"}.get(kind, "radial")
            if kind != PAINT_SOLID:
                assert len(rec["stops"]) == p.stop_count[pi]


def test_records_are_independent_of_later_scene_edits():
    sc = synth.mixed_scene(1, 96, 96)
    p = pack_scene(sc)
    g = unflatten_grads(sc, p, _filled(p, 1))
    kinds = [d.geometry["kind"] for d in unflatten_grads(sc, p, _filled(p, 1)).shapes]
    sc.shapes.reverse()  # the records come from the packed arrays, not the live scene
    assert [d.geometry["kind"] for d in g.shapes] == kinds


def test_lazy_list_behaves_like_a_list():
    made = []
    lst = LazyList(5, lambda i: made.append(i) or i * 10)
    assert made == [] and len(lst) == 5
    assert lst[-1] == 40 and lst[4] is lst[-1] and made == [4]
    assert lst[1:4] == [10, 20, 30]
    assert list(lst) == [0, 10, 20, 30, 40]
    assert sorted(made) == [0, 1, 2, 3, 4]
    with pytest.raises(IndexError):
        lst[5]
    with pytest.raises(IndexError):
        lst[-6]
