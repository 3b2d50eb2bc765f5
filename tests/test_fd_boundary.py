"""Boundary-sampled gradients against finite differences, in expectation.

Without prefiltering a pixel sample is either inside a fill or not, so the control
points and the transforms of a filled path receive gradient only from the boundary
term (edge samples drawn in proportion to length, colour jump over the pdf,
src/backward/boundary.rs:113-1148).  Its expectation over the edge samples is the
derivative of the expected image: the image averaged over the jitter of the pixel
samples.

Left: the mean of 64 runs with Philox4x32-10 boundary seeds (W*H edge samples each)
and its standard error.  Right: central finite differences of L = sum(d_render *
image) in f64, with common random numbers (the same jitter seed on both sides of a
difference), averaged over 256 jitter seeds, and their standard error.  Steps: 0.1
pixel for points and translations, 0.1 pixel / 64 for the linear entries of the
transforms (they move points up to ~64 px from the canvas centre about which the
transforms are built).  Bar, as for the Philox-against-PCG32 test: per element
z = |left - right| / sqrt(se_left^2 + se_right^2); at least 97 % of the elements
within 3 sigma, none beyond 6 sigma, mean z^2 <= 2.

Scenes: the 128x128, 4x4-spp adjoint-verification scene as generated (identity
transforms) for every control point of its four filled cubic paths, and the same
scene with rotations and translations on every shape and group for the six affine
entries of those paths' shape and group transforms.

Crate behaviour kept for parity and measured here instead: the edge term gives a
transformed shape's control points the canvas-space normal (render_edge_sample passes
it to accumulate_boundary_gradient, src/backward/boundary.rs:882-967, 970-1148), not
its pull-back to shape space, so under rotations their gradients are biased (the z
scores of the rotated scene's control points are far from the 3-sigma bar).  Also left
out: the projective row of the transforms (the forward applies them as affine maps,
the adjoint differentiates a projective one) and the stroked paths (the crate's edge
term samples the stroke bodies but not their round join and cap arcs).
"""
import numpy as np
import pytest

from dvg import BackwardOptions, RenderOptions, Rng, synth
from test_fd import _rigid_transforms

pytestmark = pytest.mark.gpu

PHILOX_SEEDS = 64
JITTER_SEEDS = 256
H_PX = 0.1


def _opts(seed):
    return RenderOptions(samples_x=4, samples_y=4, seed=seed, jitter=True, use_prefiltering=False)


def _params(sc, points=True, xforms=True):
    """(array, flat index, getter, setter, h) for the filled cubic paths."""
    from dvg import Mat3
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


def _z_scores(r, sc, params):
    """Per parameter: |mean boundary-sampled gradient - mean finite difference| over the
    combined standard error (see the module docstring)."""
    import torch

    target_sc = synth.adjoint_scene(1, sc.width, sc.height)
    target = r.render(target_sc, _opts(0)).pixels
    img = r.render(sc, _opts(0)).pixels
    dr = (2.0 * (img - target)).astype(np.float32)
    dr_dev = torch.from_numpy(dr.reshape(-1).astype(np.float64)).cuda()
    left = {}
    for b in range(PHILOX_SEEDS):
        g = r.render_backward(sc, _opts(0), BackwardOptions(rng=Rng.PHILOX, boundary_seed=1000 + b,
                                                             boundary_samples=sc.width * sc.height), dr).buffers
        for name, idx, _, _, _ in params:
            left.setdefault((name, idx), []).append(float(g[name][idx]))
    z = []
    for name, idx, get, put, h in params:
        v = get()
        hp, hm = float(np.float32(v + h)), float(np.float32(v - h))
        put(hp)
        lp = _losses(r, sc, dr_dev, JITTER_SEEDS)
        put(hm)
        lm = _losses(r, sc, dr_dev, JITTER_SEEDS)
        put(v)
        fd = (lp - lm) / (hp - hm)
        a = np.asarray(left[(name, idx)])
        se = np.sqrt(a.var(ddof=1) / a.size + fd.var(ddof=1) / fd.size)
        diff = abs(a.mean() - fd.mean())
        if se == 0.0:
            assert diff == 0.0, (name, idx)
            continue
        z.append(diff / se)
    return np.asarray(z)


def _assert_within_3_sigma(z, at_least):
    assert z.size >= at_least
    assert float(np.mean(z <= 3.0)) >= 0.97, f"{int(np.sum(z > 3.0))} of {z.size} beyond 3 sigma"
    assert float(np.max(z)) <= 6.0, f"max z {float(np.max(z)):.2f}"
    assert float(np.mean(z * z)) <= 2.0, f"mean z^2 {float(np.mean(z * z)):.2f}"


def test_cuda_boundary_point_gradients_match_fd_in_expectation():
    from dvg import Renderer

    r = Renderer(0)
    try:
        sc = synth.adjoint_scene(0, 128, 128)
        _assert_within_3_sigma(_z_scores(r, sc, _params(sc, points=True, xforms=False)), 100)
    finally:
        r.close()


def test_cuda_boundary_transform_gradients_match_fd_in_expectation():
    from dvg import Renderer

    r = Renderer(0)
    try:
        sc = _rigid_transforms(synth.adjoint_scene(0, 128, 128))
        _assert_within_3_sigma(_z_scores(r, sc, _params(sc, points=False, xforms=True)), 40)
    finally:
        r.close()


def test_cuda_boundary_points_of_rotated_shapes_measured_exclusion():
    """The crate's canvas-space normal on shape-space control points: on the rotated
    scene the control points' z scores are far outside the bar the untransformed scene
    meets (mean z^2 well above 2)."""
    from dvg import Renderer

    r = Renderer(0)
    try:
        sc = _rigid_transforms(synth.adjoint_scene(0, 128, 128))
        z = _z_scores(r, sc, _params(sc, points=True, xforms=False)[::3])
        assert float(np.mean(z * z)) > 4.0, f"mean z^2 {float(np.mean(z * z)):.2f}"
    finally:
        r.close()
