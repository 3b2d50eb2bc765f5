"""Host-side scene packing: the native packer (csrc/pack.cpp, `dvg.abi.pack_scene`)
against the plain-Python reference (`dvg.abi.pack_scene_python`), byte for byte, on
every synthetic workload and on inputs that take the packers' conversion paths
(float64 points and matrices, numpy indices, per-point thickness, empty scenes)."""
import numpy as np
import pytest

from dvg import abi, synth
from dvg.scene import Color, GradientStop, LinearGradient, Mat3, Scene, ShapeGroup, StrokeCap, StrokeJoin


def _same(a, b):
    assert a.arrays.keys() == b.arrays.keys()
    for k in a.arrays:
        x, y = a.arrays[k], b.arrays[k]
        assert x.dtype == y.dtype and x.shape == y.shape, k
        assert x.tobytes() == y.tobytes(), k
    for f, _ in abi.SceneDesc._fields_:
        va, vb = getattr(a.desc, f), getattr(b.desc, f)
        if isinstance(va, (int, float)):
            assert va == vb, f
        elif f == "background":
            assert list(va) == list(vb)
        else:  # pointers: both set or both null
            assert bool(va) == bool(vb), f
    assert a.paint_of == b.paint_of
    assert a.path_point_offset == b.path_point_offset and a.path_point_count == b.path_point_count
    assert a.stop_offset == b.stop_offset and a.stop_count == b.stop_count


def _converted_scene():
    sc = synth.plain_scene(5, 64, 64, 6)
    sc.shapes[0].geometry.path.thickness = [0.5 + 0.1 * i for i in range(3)]  # shorter than the points
    sc.shapes[1].geometry.path.points = np.asarray(sc.shapes[1].geometry.path.points, np.float64)
    sc.shapes[2].transform.m = np.asarray(sc.shapes[2].transform.m, np.float64)
    sc.shapes[3].transform = Mat3.rotate(0.7)
    sc.shapes[3].stroke_join = StrokeJoin.MITER
    sc.shapes[3].stroke_cap = StrokeCap.SQUARE
    sc.shapes[3].stroke_width = np.float32(2.5)
    sc.groups[0].shape_indices = np.asarray(sc.groups[0].shape_indices, np.int32)
    sc.groups.append(ShapeGroup([4, 5], None,
                                LinearGradient((0.0, 0.0), (9.0, 3.0), [GradientStop(0.25, Color(1, 0, 0, 1))])))
    return sc


@pytest.mark.parametrize("make", [
    lambda: synth.mixed_scene(0), lambda: synth.mixed_scene(7, 96, 80, scale=0.2),
    lambda: synth.plain_scene(3, 64, 64, 8), synth.primitives_scene, lambda: synth.styled_stroke_scene(1),
    lambda: synth.adjoint_scene(0), lambda: synth.large_scene(0), lambda: Scene(16, 16), lambda: Scene(0, 8),
    _converted_scene,
])
def test_native_packer_matches_python(make):
    sc = make()
    _same(abi.pack_scene(sc), abi.pack_scene_python(sc))


def test_packers_reject_the_same_inputs():
    class Odd:
        pass

    sc = synth.plain_scene(1, 16, 16, 2)
    sc.shapes[0].geometry = Odd()
    for pack in (abi.pack_scene, abi.pack_scene_python):
        with pytest.raises(TypeError):
            pack(sc)
    sc = synth.plain_scene(1, 16, 16, 2)
    sc.groups[0].fill = "red"
    for pack in (abi.pack_scene, abi.pack_scene_python):
        with pytest.raises(TypeError):
            pack(sc)
