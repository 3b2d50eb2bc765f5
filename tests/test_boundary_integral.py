"""The oracle's deterministic boundary integral (oracle_boundary_integral), the
reference the GPU boundary estimator is checked against in expectation
(tests/test_fd_boundary.py), pinned on the CPU:

- it is the mean of the oracle's own boundary passes over Philox seeds (which follow
  the crate's render_backward sample by sample), on a small adjoint scene;
- the crate's colour-sampling offset (1e-4 of the canvas along the normal,
  src/backward/boundary.rs:880-902) shifts the integral where an edge crosses another
  colour edge: on the adjoint scene, whose filled paths cross each other and the
  strokes, some control-point gradients move by more than 5 % between the crate's
  offset and one 128 times smaller; on four separated outlines they agree to 1e-3.
"""
import numpy as np

from dvg import BackwardOptions, RenderOptions, Rng, synth
from test_fd_boundary import separated_blobs


def _opts(seed=0):
    return RenderOptions(samples_x=4, samples_y=4, seed=seed, jitter=True, use_prefiltering=False)


def _d_render(sc, target_sc):
    import pyoracle

    return (2.0 * (pyoracle.render(sc, _opts()) - pyoracle.render(target_sc, _opts()))).astype(np.float32)


def test_oracle_integral_is_the_mean_of_boundary_passes():
    import pyoracle

    sc, tsc = synth.adjoint_scene(0, 48, 48), synth.adjoint_scene(1, 48, 48)
    dr = _d_render(sc, tsc)
    names = ("d_points", "d_shape_stroke_width", "d_shape_transform", "d_group_transform")
    runs = {n: [] for n in names}
    for b in range(256):
        _, buf = pyoracle.render_backward(sc, _opts(), BackwardOptions(rng=Rng.PHILOX, boundary_seed=b), dr,
                                          passes=2, threads=8)
        for n in names:
            runs[n].append(np.asarray(buf[n], np.float64).copy())
    _, integral = pyoracle.boundary_integral(sc, _opts(), dr, 400_000)
    z = []
    for n in names:
        a = np.asarray(runs[n])
        ref = np.asarray(integral[n], np.float64)
        se = np.sqrt(a.var(0, ddof=1) / a.shape[0] + (1e-3 * np.abs(ref)) ** 2)
        live = se > 0
        assert np.all(np.abs(a.mean(0) - ref)[~live] <= 1e-6), n
        z.append(np.abs(a.mean(0) - ref)[live] / se[live])
    z = np.concatenate(z)
    assert z.size >= 100
    assert float(np.mean(z <= 3.0)) >= 0.97, f"{int(np.sum(z > 3.0))} of {z.size} beyond 3 sigma"
    assert float(np.max(z)) <= 6.0
    assert float(np.mean(z * z)) <= 2.0


def _offset_shift(sc, tsc):
    """Relative change of the filled paths' control-point gradients between the crate's
    colour offset and one 128 times smaller."""
    import pyoracle

    dr = _d_render(sc, tsc)
    _, crate = pyoracle.boundary_integral(sc, _opts(), dr, 400_000, 1.0e-4)
    _, fine = pyoracle.boundary_integral(sc, _opts(), dr, 400_000, 1.0e-4 / 128)
    a, b = np.asarray(crate["d_points"], np.float64), np.asarray(fine["d_points"], np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-2 * np.abs(b).max())


def test_colour_offset_shifts_gradients_only_where_edges_cross():
    sc = synth.adjoint_scene(0, 128, 128)
    filled = 2 * sum(len(s.geometry.path.points) for s in sc.shapes if s.stroke_width == 0)
    shift = _offset_shift(sc, synth.adjoint_scene(1, 128, 128))[:filled]
    assert float(shift.max()) > 0.05, f"largest shift {float(shift.max()):.4f}"
    assert int(np.sum(shift > 0.02)) >= 3
    assert float(_offset_shift(separated_blobs(seed=0), separated_blobs(seed=1)).max()) < 1e-3
