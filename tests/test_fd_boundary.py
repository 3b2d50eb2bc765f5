"""Boundary-sampled gradients in expectation.

Without prefiltering a pixel sample is either inside a fill or not, so the control
points, stroke widths and transforms receive gradient only from the boundary term
(edge samples drawn in proportion to length, colour jump over the pdf,
src/backward/boundary.rs:113-1148).  Two checks of its expectation over boundary seeds:

1. Against the crate's own integral.  The oracle's boundary_integral takes the edge
   term of every boundary point of every shape (midpoint rule over the boundary
   parameter, the same per-point evaluation as a drawn sample), which is what the
   crate's boundary gradients average to over seeds.  Left: the mean of 128 runs with
   Philox4x32-10 seeds (W*H edge samples each) and its standard error.  Scenes: the
   128x128, 4x4-spp adjoint-verification scene as generated (four filled cubic paths
   that cross themselves and each other, four stroked quadratic paths) and the same
   scene with rotations and translations on every shape and group; every control
   point, stroke width and affine transform entry.

2. Against finite differences of the rendered image.  Right: central differences of
   L = sum(d_render * image) in f64 with common random numbers (the same jitter seed
   on both sides), averaged over 256 jitter seeds.  Steps: 0.1 pixel for points and
   translations, 0.1 pixel / 64 for the linear transform entries, whose differences are
   extrapolated from h and h/2 (Richardson) to cancel their h^2 term.  Scene: four smooth
   closed cubic outlines, one per quadrant, whose boundaries cross neither themselves
   nor each other (see below), untransformed for the control points and rotated about
   their own centres for the transform entries.

Bar for both: per element z = |left - right| / (combined standard error); at least
97 % of the elements within 3 sigma, none beyond 6 sigma, mean z^2 <= 2.

Crate behaviour kept for parity, measured here instead of passed over:
- The colours either side of an edge point are sampled 1e-4 of the canvas size away
  along the normal (render_edge_sample, boundary.rs:880-902; 0.0128 px on 128x128).
  Where the edge crosses another colour edge at a shallow angle, both offset points
  straddle that edge too for a stretch of about 2 * offset / sin(angle), and the term
  picks up the other edge's colour jump there.  The crossings of the adjoint scene
  move its control-point gradients by up to ~12 % from the derivative of the image,
  which is why the finite-difference check runs on a scene without crossings
  (tests/test_boundary_integral.py measures the offset's effect on both scenes).
- The edge term gives a transformed shape's control points the canvas-space normal
  (render_edge_sample passes it to accumulate_boundary_gradient, boundary.rs:882-967,
  970-1148), not its pull-back to shape space: under rotations their gradients are
  biased (the last test measures it against finite differences).
Also outside the finite-difference check: the projective row of the transforms (the
forward applies them as affine maps, the adjoint differentiates a projective one).
"""
import numpy as np
import pytest

from dvg import BackwardOptions, Color, Filter, FilterType, Mat3, Path, PathGeometry, RenderOptions, Rng, Scene, \
    Shape, ShapeGroup, synth
from test_fd import _rigid_transforms

pytestmark = pytest.mark.gpu

PHILOX_SEEDS = 64
INTEGRAL_SEEDS = 128
JITTER_SEEDS = 256
H_PX = 0.1
INTEGRAL_STEPS = 400_000  # midpoint steps of each shape's boundary parameter
INTEGRAL_REL = 1e-3  # allowance for the midpoint rule, relative to the integral


def _opts(seed):
    return RenderOptions(samples_x=4, samples_y=4, seed=seed, jitter=True, use_prefiltering=False)


def separated_blobs(width=128, height=128, seed=0):
    """Four smooth closed cubic outlines (5-7 segments about a circle of radius 0.3 of
    a quadrant, tangent handles of a third of the chord), one per quadrant, opaque or
    semi-transparent solid fills: no boundary crosses another or itself."""
    rng = np.random.default_rng(seed)
    sc = Scene(width, height)
    sc.background = Color(1.0, 1.0, 1.0, 1.0)
    sc.filter = Filter(FilterType.BOX, 0.5)
    r0 = 0.3 * min(width, height) / 2
    for qy in range(2):
        for qx in range(2):
            c = np.array([(qx + 0.5) * width / 2, (qy + 0.5) * height / 2])
            n = int(rng.integers(5, 8))
            ang = 2 * np.pi * (np.arange(n) + rng.uniform(-0.2, 0.2, n)) / n
            rad = r0 * (1.0 + rng.uniform(-0.2, 0.2, n))
            a = c + rad[:, None] * np.stack([np.cos(ang), np.sin(ang)], 1)
            tan = np.stack([-np.sin(ang), np.cos(ang)], 1)
            pts = []
            for k in range(n):
                k1 = (k + 1) % n
                hl = np.linalg.norm(a[k1] - a[k]) / 3.0
                pts += [a[k], a[k] + hl * tan[k], a[k1] - hl * tan[k1]]
            pts = np.asarray(pts, np.float32)
            sc.shapes.append(Shape(PathGeometry(Path([2] * n, [tuple(map(float, p)) for p in pts], None, True,
                                                     False))))
            rgb = np.float32(rng.uniform(0.0, 1.0, 3))
            alpha = float(rng.choice([1.0, 0.6]))
            sc.groups.append(ShapeGroup([len(sc.shapes) - 1], Color(*map(float, rgb), alpha), None))
    return sc


def _rigid_about_centres(sc):
    """Each shape rotated about its own centre and moved by a pixel or two; each group
    rotated the other way about the same centre: no two outlines come to cross."""
    for i, (s, g) in enumerate(zip(sc.shapes, sc.groups)):
        c = np.mean(np.asarray(s.geometry.path.points, np.float64), 0)
        s.transform = Mat3.translate(*c).mul(Mat3.rotate(0.3 * (i + 1))).mul(Mat3.translate(*(-c)))
        g.set_shape_to_canvas(Mat3.translate(1.5 - 0.5 * i, -1.0 + 0.5 * i).mul(Mat3.translate(*c)).mul(
            Mat3.rotate(-0.2 * (i + 1))).mul(Mat3.translate(*(-c))))
    return sc


def _params(sc, points=True, xforms=True):
    """(array, flat index, getter, setter, h) for the filled cubic paths."""
    from dvg.abi import pack_scene

    packed = pack_scene(sc)
    out = []
    for si, shp in enumerate(sc.shapes):
        path = shp.geometry.path
        if shp.stroke_width > 0 or max(path.num_control_points) < 2:
            continue
        base = packed.path_point_offset[si]
        for k in range(len(path.points) if points else 0):
            for c in range(2):
                def get(path=path, k=k, c=c):
                    return path.points[k][c]

                def put(v, path=path, k=k, c=c):
                    p = list(path.points[k])
                    p[c] = v
                    path.points[k] = tuple(p)
                out.append(("d_points", 2 * (base + k) + c, get, put, H_PX))
        gi = next(i for i, g in enumerate(sc.groups) if si in g.shape_indices)
        for k in range(6 if xforms else 0):
            h = H_PX if k in (2, 5) else H_PX / 64.0

            def sget(s=shp, k=k):
                return float(s.transform.m.reshape(-1)[k])

            def sput(v, s=shp, k=k):
                m = s.transform.m.reshape(-1).copy()
                m[k] = v
                s.transform = Mat3(m)

            def gget(g=sc.groups[gi], k=k):
                return float(g.shape_to_canvas.m.reshape(-1)[k])

            def gput(v, g=sc.groups[gi], k=k):
                m = g.shape_to_canvas.m.reshape(-1).copy()
                m[k] = v
                g.set_shape_to_canvas(Mat3(m))
            out.append(("d_shape_transform", 9 * si + k, sget, sput, h))
            out.append(("d_group_transform", 9 * gi + k, gget, gput, h))
    return out


def _losses(r, sc, dr, n_seeds):
    """L_s = sum(d_render * image_s) in f64 for the jitter seeds 0..n_seeds-1 (device renders)."""
    import torch

    up = r.upload(sc)
    npx = sc.width * sc.height * 4
    imgs = torch.empty((n_seeds, npx), device="cuda")
    torch.cuda.synchronize()
    for s in range(n_seeds):
        up.render_device(_opts(s), imgs[s].data_ptr())
    torch.cuda.synchronize()
    up.close()
    return (imgs.double() @ dr).cpu().numpy()


def _d_render(r, sc, target_sc):
    target = r.render(target_sc, _opts(0)).pixels
    img = r.render(sc, _opts(0)).pixels
    return (2.0 * (img - target)).astype(np.float32)


def _boundary_runs(r, sc, dr, names, n_seeds):
    """Boundary-sampled gradients of n_seeds Philox seeds: {name: (n_seeds, size)}."""
    runs = {n: [] for n in names}
    for b in range(n_seeds):
        g = r.render_backward(sc, _opts(0), BackwardOptions(rng=Rng.PHILOX, boundary_seed=1000 + b,
                                                             boundary_samples=sc.width * sc.height), dr).buffers
        for n in names:
            runs[n].append(np.asarray(g[n], np.float64).copy())
    return {n: np.asarray(v) for n, v in runs.items()}


def _central(r, sc, dr_dev, get, put, h):
    """Central differences per jitter seed (common random numbers on both sides)."""
    v = get()
    hp, hm = float(np.float32(v + h)), float(np.float32(v - h))
    put(hp)
    lp = _losses(r, sc, dr_dev, JITTER_SEEDS)
    put(hm)
    lm = _losses(r, sc, dr_dev, JITTER_SEEDS)
    put(v)
    return (lp - lm) / (hp - hm)


def _z_scores_fd(r, sc, target_sc, params, richardson=False):
    """Per parameter: |mean boundary-sampled gradient - mean finite difference| over the
    combined standard error (see the module docstring).  richardson: (4 D(h/2) - D(h)) / 3
    per jitter seed, which cancels the h^2 term of the central differences D (the
    transforms' linear entries move points far from the origin by up to 0.15 px at h,
    where that term reaches ~10 % of some entries)."""
    import torch

    dr = _d_render(r, sc, target_sc)
    dr_dev = torch.from_numpy(dr.reshape(-1).astype(np.float64)).cuda()
    runs = _boundary_runs(r, sc, dr, sorted({p[0] for p in params}), PHILOX_SEEDS)
    z = []
    for name, idx, get, put, h in params:
        fd = _central(r, sc, dr_dev, get, put, h)
        if richardson:
            fd = (4.0 * _central(r, sc, dr_dev, get, put, h / 2) - fd) / 3.0
        a = runs[name][:, idx]
        se = np.sqrt(a.var(ddof=1) / a.size + fd.var(ddof=1) / fd.size)
        diff = abs(a.mean() - fd.mean())
        if se == 0.0:
            assert diff == 0.0, (name, idx)
            continue
        z.append(diff / se)
    return np.asarray(z)


def _z_scores_integral(r, sc, target_sc, names):
    """Per gradient element: |mean boundary-sampled gradient - the oracle's integral of
    the crate's edge term| over the standard error of the mean (plus the integral's
    allowance)."""
    import pyoracle

    dr = _d_render(r, sc, target_sc)
    runs = _boundary_runs(r, sc, dr, names, INTEGRAL_SEEDS)
    _, integral = pyoracle.boundary_integral(sc, _opts(0), dr, INTEGRAL_STEPS)
    z = []
    for n in names:
        a = runs[n]
        ref = np.asarray(integral[n], np.float64)[: a.shape[1]]
        se = np.sqrt(a.var(0, ddof=1) / a.shape[0] + (INTEGRAL_REL * np.abs(ref)) ** 2)
        diff = np.abs(a.mean(0) - ref)
        live = se > 0.0
        assert np.all(diff[~live] <= 1e-6 * max(1.0, float(np.abs(ref).max()))), n
        z.append(diff[live] / se[live])
    return np.concatenate(z)


def _assert_within_3_sigma(z, at_least):
    assert z.size >= at_least
    assert float(np.mean(z <= 3.0)) >= 0.97, f"{int(np.sum(z > 3.0))} of {z.size} beyond 3 sigma"
    assert float(np.max(z)) <= 6.0, f"max z {float(np.max(z)):.2f}"
    assert float(np.mean(z * z)) <= 2.0, f"mean z^2 {float(np.mean(z * z)):.2f}"


INTEGRAL_NAMES = ("d_points", "d_shape_stroke_width", "d_shape_transform", "d_group_transform")


@pytest.mark.parametrize("rotated", [False, True], ids=["as generated", "rotated"])
def test_cuda_boundary_gradients_match_crate_integral(rotated):
    from dvg import Renderer

    r = Renderer(0)
    try:
        sc = synth.adjoint_scene(0, 128, 128)
        if rotated:
            sc = _rigid_transforms(sc)
        _assert_within_3_sigma(_z_scores_integral(r, sc, synth.adjoint_scene(1, 128, 128), INTEGRAL_NAMES), 250)
    finally:
        r.close()


def test_cuda_boundary_point_gradients_match_fd_in_expectation():
    from dvg import Renderer

    r = Renderer(0)
    try:
        sc = separated_blobs(seed=0)
        _assert_within_3_sigma(_z_scores_fd(r, sc, separated_blobs(seed=1), _params(sc, points=True, xforms=False)),
                               100)
    finally:
        r.close()


def test_cuda_boundary_transform_gradients_match_fd_in_expectation():
    from dvg import Renderer

    r = Renderer(0)
    try:
        sc = _rigid_about_centres(separated_blobs(seed=0))
        _assert_within_3_sigma(_z_scores_fd(r, sc, separated_blobs(seed=1), _params(sc, points=False, xforms=True),
                                            richardson=True), 40)
    finally:
        r.close()


def test_cuda_boundary_points_of_rotated_shapes_measured_exclusion():
    """The crate's canvas-space normal on shape-space control points: on the rotated
    outlines the control points' z scores against finite differences are far outside
    the bar the untransformed outlines meet (mean z^2 well above 2)."""
    from dvg import Renderer

    r = Renderer(0)
    try:
        sc = _rigid_about_centres(separated_blobs(seed=0))
        z = _z_scores_fd(r, sc, separated_blobs(seed=1), _params(sc, points=True, xforms=False)[::3])
        assert float(np.mean(z * z)) > 4.0, f"mean z^2 {float(np.mean(z * z)):.2f}"
    finally:
        r.close()
