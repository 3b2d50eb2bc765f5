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

from dvg import BackwardOptions, Color, RenderOptions, synth
from dvg.abi import pack_scene

H_PAINT = 1e-3
H_POINT = 2.5e-3
RTOL_DEFAULT = 1e-4
ATOL = 1e-5


def _params(sc, prefilter, bg_alpha=True, h_paint=H_PAINT, h_point=H_POINT):
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
    return out


def _check(sc, opts, render, backward, bg_alpha=True, h_paint=H_PAINT, h_point=H_POINT, point_rtol=1e-3):
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

    for name, idx, get, put, h in _params(sc, opts.use_prefiltering, bg_alpha, h_paint, h_point):
        fd.setdefault(name, []).append((idx, central(get, put, h)))
    for name, pairs in fd.items():
        g = np.asarray(grads[name], np.float64)
        idx = np.array([i for i, _ in pairs])
        f = np.array([x for _, x in pairs])
        scale = float(np.max(np.abs(g[idx])))
        err = float(np.max(np.abs(g[idx] - f)))
        rtol = point_rtol if name == "d_points" else RTOL_DEFAULT
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


@pytest.mark.gpu
@pytest.mark.parametrize("prefilter", [False, True])
def test_cuda_interior_gradients_match_fd(prefilter):
    from dvg import Renderer

    sc = synth.adjoint_scene(0, 128, 128)
    opts = RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=not prefilter, use_prefiltering=prefilter)
    r = Renderer(0)
    try:
        def render(sc, opts):
            return r.render(sc, opts).pixels

        def backward(sc, opts, b, dr):
            return r.render_backward(sc, opts, b, dr).buffers

        _check(sc, opts, render, backward, bg_alpha=False, h_paint=1e-2, h_point=2.5e-3, point_rtol=2e-3)
    finally:
        r.close()
