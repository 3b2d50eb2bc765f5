"""Interior gradients against central finite differences.

Loss L = sum(d_render * image), accumulated in f64 from the f32 render; the
analytic gradient is render_backward with the same d_render.  FD step h = 1e-3 on
paint, background and stroke-width parameters, bar: per gradient array,
max |analytic - FD| <= 1e-4 * max |analytic| + 1e-5.  Line / quadratic control
points (prefiltered mode) use h = 2.5e-3 with a bar of 1e-3 * max |analytic|:
the render is f32 (the crate's arithmetic), whose rounding gives these
differences a noise floor of a few 1e-4 of the gradient scale (~1e-3 at
h = 1e-3), while steps of 1e-2 already cross the C1 edges of the smoothstep
coverage on some samples.  The perturbation
actually applied is float32(v + h) - float32(v - h).

Transforms (prefiltered): the six affine entries of every stroke shape's transform
and of its group's shape_to_canvas, under rotations and translations
(test_oracle_transform_gradients_match_fd, and the GPU case with xforms); the
projective row, non-uniform scales and cubic points are measured exclusions
(test_measured_crate_adjoint_exclusions).  Boundary-sampled (non-prefiltered)
control points and transforms are checked in expectation in
tests/test_fd_boundary.py.

Cubic control points in prefiltered mode are left out: the crate's cubic
closest-point adjoint (src/backward/distance.rs:292-391, restated by the oracle
and by the CUDA path) drops the dD/dp3 term and half of d(2 b.b)/dp, so it is not
the derivative of its own forward pass (measured: up to 4 % of the gradient scale
on 48x48 scenes); parity with the crate is kept there and checked in the parity
tests instead.

What render_backward differentiates is the crate's CPU image: per pixel, the
filter-weighted average of per-sample colours that are un-premultiplied per
sample (src/backward/sampling.rs:76-224, src/backward/filters.rs:70-103); the
forward image un-premultiplies once per pixel after the splat
(src/gpu/kernels/forward.rs:294-334).  The two agree wherever every sample of a
pixel is opaque.  So the CPU tests difference oracle.render_differentiated (all
parameters, opaque and translucent backgrounds) and the GPU test differences the
CUDA forward image on an opaque background, leaving out the background alpha
(the one parameter that changes a sample's final alpha there).  A translucent
background is checked without prefiltering only: with prefiltering the crate
returns the premultiplied background for a sample with no fragment and the
un-premultiplied colour as soon as one fragment has non-zero coverage, a jump
that finite differences see and the adjoint (rightly) does not.

CPU: the oracle on a 48x48, 2x2-spp adjoint scene.  GPU: the CUDA path on the
128x128, 4x4-spp adjoint-verification scene, with h = 1e-2 on paint, background
and stroke-width parameters: over 16 k pixels the f32 rounding of the render
alone moves an h = 1e-3 difference by ~1e-4 of the gradient scale (measured
1.1e-4), while the image is linear in the colour channels, so the larger step
adds no truncation error there.  Control points keep h = 2.5e-3 with a bar of
2e-3 of the scale: with 16 samples per pixel the smoothstep coverage puts C1 edges
within 1e-2 of many samples, so larger steps carry truncation error (measured on
the oracle: 1.4e-3 of the scale at h = 5e-3, 2e-4 at h = 1.25e-3), smaller ones the
f32 noise.
"""
import numpy as np
import pytest

from dvg import BackwardOptions, Color, Mat3, RenderOptions, synth
from dvg.abi import pack_scene

H_PAINT = 1e-3
H_POINT = 2.5e-3
H_XLIN = 1e-4  # linear transform entries multiply coordinates of ~20-100 px
RTOL_DEFAULT = 1e-4
ATOL = 1e-5
GEOMETRIC = ("d_points", "d_shape_transform", "d_group_transform")


def _rigid_transforms(sc):
    """Rotations and translations about the canvas centre on every shape and group
    (the transforms whose adjoint the crate gets right; see the measured exclusions
    below)."""
    c = sc.width / 2.0
    for i, s in enumerate(sc.shapes):
        s.transform = Mat3.translate(c, c).mul(Mat3.rotate(0.15 * (i + 1))).mul(Mat3.translate(-c, -c))
    for i, g in enumerate(sc.groups):
        g.set_shape_to_canvas(Mat3.translate(1.5 - 0.3 * i, -1.0 + 0.2 * i).mul(Mat3.translate(c, c)).mul(
            Mat3.rotate(-0.1 * i)).mul(Mat3.translate(-c, -c)))
    return sc


def _xform_param(name, owner, attr, index, k, h, regroup=False):
    """Entry k of a Mat3 attribute; a group's canvas_to_shape follows its shape_to_canvas."""
    def get():
        return float(getattr(owner, attr).m.reshape(-1)[k])

    def put(v):
        m = getattr(owner, attr).m.reshape(-1).copy()
        m[k] = v
        if regroup:
            owner.set_shape_to_canvas(Mat3(m))
        else:
            setattr(owner, attr, Mat3(m))
    return (name, 9 * index + k, get, put, h)


def _params(sc, prefilter, bg_alpha=True, h_paint=H_PAINT, h_point=H_POINT, xforms=False):
    """(array name, flat index, getter, setter, h) for every checked parameter."""
    packed = pack_scene(sc)
    out = []
    for (gi, which), pi in packed.paint_of.items():
        paint = getattr(sc.groups[gi], which)
        if isinstance(paint, Color):
            for c, ch in enumerate("rgba"):
                out.append(("d_paint_params", 4 * pi + c,
                            lambda p=paint, ch=ch: getattr(p, ch),
                            lambda v, p=paint, ch=ch: setattr(p, ch, v), h_paint))
    for c, ch in enumerate("rgba" if bg_alpha else "rgb"):
        out.append(("d_background", c, lambda ch=ch: getattr(sc.background, ch),
                    lambda v, ch=ch: setattr(sc.background, ch, v), h_paint))
    if prefilter:
        for si, shp in enumerate(sc.shapes):
            if shp.stroke_width > 0:
                out.append(("d_shape_stroke_width", si, lambda s=shp: s.stroke_width,
                            lambda v, s=shp: setattr(s, "stroke_width", v), h_paint))
            path = shp.geometry.path
            if max(path.num_control_points) < 2:  # lines and quadratics only
                base = packed.path_point_offset[si]
                for k in range(len(path.points)):
                    for c in range(2):
                        def get(path=path, k=k, c=c):
                            return path.points[k][c]

                        def put(v, path=path, k=k, c=c):
                            p = list(path.points[k])
                            p[c] = v
                            path.points[k] = tuple(p)
                        out.append(("d_points", 2 * (base + k) + c, get, put, h_point))
                if xforms:  # the affine entries of the shape's and its group's transforms
                    gi = next(i for i, g in enumerate(sc.groups) if si in g.shape_indices)
                    for k in range(6):
                        h = h_point if k in (2, 5) else H_XLIN
                        out.append(_xform_param("d_shape_transform", shp, "transform", si, k, h))
                        out.append(_xform_param("d_group_transform", sc.groups[gi], "shape_to_canvas", gi, k, h,
                                                regroup=True))
    return out


def _check(sc, opts, render, backward, bg_alpha=True, h_paint=H_PAINT, h_point=H_POINT, point_rtol=1e-3,
           xforms=False, xform_rtol=5e-3):
    img = render(sc, opts)
    rng = np.random.default_rng(5)
    target = np.clip(img + rng.normal(0, 0.1, img.shape).astype(np.float32), 0, 1)
    dr = (2.0 * (img - target)).astype(np.float32)
    grads = backward(sc, opts, BackwardOptions(boundary_samples=1), dr)
    dr64 = dr.astype(np.float64)
    fd = {}
    def central(get, put, h):
        v = get()
        hp, hm = float(np.float32(v + h)), float(np.float32(v - h))
        put(hp)
        lp = float(np.sum(render(sc, opts).astype(np.float64) * dr64))
        put(hm)
        lm = float(np.sum(render(sc, opts).astype(np.float64) * dr64))
        put(v)
        return (lp - lm) / (hp - hm)

    for name, idx, get, put, h in _params(sc, opts.use_prefiltering, bg_alpha, h_paint, h_point, xforms):
        fd.setdefault(name, []).append((idx, central(get, put, h)))
    for name, pairs in fd.items():
        g = np.asarray(grads[name], np.float64)
        idx = np.array([i for i, _ in pairs])
        f = np.array([x for _, x in pairs])
        scale = float(np.max(np.abs(g[idx])))
        err = float(np.max(np.abs(g[idx] - f)))
        # with transforms the stroke width also moves edges through the scale: geometric bar
        rtol = point_rtol if name in GEOMETRIC or (xforms and name == "d_shape_stroke_width") else RTOL_DEFAULT
        if name in ("d_shape_transform", "d_group_transform"):
            rtol = xform_rtol
        assert err <= rtol * scale + ATOL, f"{name}: max |analytic - FD| {err:.3e}, scale {scale:.3e}"
    return fd


@pytest.mark.parametrize("prefilter,translucent", [(False, False), (False, True), (True, False)])
def test_oracle_interior_gradients_match_fd(prefilter, translucent):
    import pyoracle

    sc = synth.adjoint_scene(0, 48, 48)
    if translucent:
        sc.background = Color(0.3, 0.5, 0.7, 0.6)
    opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=not prefilter, use_prefiltering=prefilter)

    def backward(sc, opts, b, dr):
        return pyoracle.render_backward(sc, opts, b, dr)[1]

    fd = _check(sc, opts, pyoracle.render_differentiated, backward)
    assert len(fd["d_paint_params"]) == 32 and len(fd["d_background"]) == 4


def test_oracle_transform_gradients_match_fd():
    """Prefiltered: shape and group transform entries (and the points, paints and
    stroke widths) of the line / quadratic strokes, under rotations, uniform scales
    and translations, against finite differences of the oracle's image."""
    import pyoracle

    sc = _rigid_transforms(synth.adjoint_scene(0, 48, 48))
    opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=False, use_prefiltering=True)

    def backward(sc, opts, b, dr):
        return pyoracle.render_backward(sc, opts, b, dr)[1]

    # geometric bar 3e-3 of the scale: the measured floor of this scene's prefiltered
    # point gradients is 1.0e-3 without transforms and up to 2.3e-3 with rotated
    # groups, the same for every step h in [1.25e-3, 1e-2] (a small systematic
    # difference, not step truncation or f32 noise).  Transform bar 5e-3: the linear
    # entries (h = 1e-4) measure 3.0e-3, growing with h (4.5e-3 at 3e-4, 8e-3 at 1e-3:
    # they move points ~50 px from the origin, so truncation dominates above 1e-4).
    fd = _check(sc, opts, pyoracle.render_differentiated, backward, point_rtol=3e-3, xforms=True)
    assert len(fd["d_shape_transform"]) == 24 and len(fd["d_group_transform"]) == 24


def _defect(sc, opts, param):
    """max |analytic - FD| / max |analytic| over the given (name, index, get, put, h) list."""
    import pyoracle

    img = pyoracle.render_differentiated(sc, opts)
    rng = np.random.default_rng(5)
    dr = (2.0 * (img - np.clip(img + rng.normal(0, 0.1, img.shape).astype(np.float32), 0, 1))).astype(np.float32)
    g = pyoracle.render_backward(sc, opts, BackwardOptions(boundary_samples=1), dr)[1]
    dr64 = dr.astype(np.float64)
    a, f = [], []
    for name, idx, get, put, h in param:
        v = get()
        put(v + h)
        lp = float(np.sum(pyoracle.render_differentiated(sc, opts).astype(np.float64) * dr64))
        put(v - h)
        lm = float(np.sum(pyoracle.render_differentiated(sc, opts).astype(np.float64) * dr64))
        put(v)
        a.append(float(g[name][idx]))
        f.append((lp - lm) / (2 * h))
    a, f = np.array(a), np.array(f)
    return float(np.max(np.abs(a - f)) / np.max(np.abs(a))), a, f


def test_measured_crate_adjoint_exclusions():
    """Where the crate's prefiltered adjoint is not the derivative of its own forward
    pass; the oracle and the CUDA path keep the crate's arithmetic (parity first), so
    these parameters are excluded from the finite-difference bars above.  Measured on
    the 48x48, 2x2-spp adjoint scene:
    * the projective row of a transform (entries 6-8): the forward applies transforms
      as affine maps (src/math.rs:198-202) while the adjoint differentiates a projective
      map (src/backward/math.rs:109-128); finite differences are exactly 0, the
      analytic values are not;
    * non-uniform scales: the closest point is found in shape space and the adjoint
      treats it as the canvas-space closest point (src/backward/distance.rs:50-136),
      off by tens of percent of the gradient scale;
    * cubic control points: the cubic closest-point adjoint drops terms
      (src/backward/distance.rs:292-391), off by a few percent."""
    opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=False, use_prefiltering=True)
    sc = _rigid_transforms(synth.adjoint_scene(0, 48, 48))
    proj = [_xform_param("d_shape_transform", sc.shapes[5], "transform", 5, k, H_XLIN) for k in (6, 7)]
    _, a, f = _defect(sc, opts, proj)
    assert np.all(f == 0.0) and np.all(np.abs(a) > 1.0)
    sc = synth.adjoint_scene(0, 48, 48)
    for s in sc.shapes:
        c = sc.width / 2.0
        s.transform = Mat3.translate(c, c).mul(Mat3.scale(0.9, 1.05)).mul(Mat3.translate(-c, -c))
    aniso = [_xform_param("d_shape_transform", sc.shapes[si], "transform", si, k, H_XLIN)
             for si in (4, 5) for k in (0, 4)]
    rel, _, _ = _defect(sc, opts, aniso)
    assert rel > 0.1
    sc = synth.adjoint_scene(0, 48, 48)
    path = sc.shapes[1].geometry.path
    base = pack_scene(sc).path_point_offset[1]

    def pt_param(k, c):
        def get():
            return path.points[k][c]

        def put(v):
            p = list(path.points[k])
            p[c] = v
            path.points[k] = tuple(p)
        return ("d_points", 2 * (base + k) + c, get, put, H_POINT)
    rel, _, _ = _defect(sc, opts, [pt_param(k, c) for k in range(len(path.points)) for c in (0, 1)])
    assert 0.005 < rel < 0.2


@pytest.mark.gpu
@pytest.mark.parametrize("prefilter,xforms", [(False, False), (True, False), (True, True)])
def test_cuda_interior_gradients_match_fd(prefilter, xforms):
    from dvg import Renderer

    sc = synth.adjoint_scene(0, 128, 128)
    if xforms:
        sc = _rigid_transforms(sc)
    opts = RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=not prefilter, use_prefiltering=prefilter)
    r = Renderer(0)
    try:
        def render(sc, opts):
            return r.render(sc, opts).pixels

        def backward(sc, opts, b, dr):
            return r.render_backward(sc, opts, b, dr).buffers

        _check(sc, opts, render, backward, bg_alpha=False, h_paint=1e-2, h_point=2.5e-3,
               point_rtol=3e-3 if xforms else 2e-3, xforms=xforms)
    finally:
        r.close()
