"""Boundary-sampled gradients in expectation.

Philox4x32-10 boundary samples averaged over 64 seeds against the expectation
of the crate's PCG32 stream over 64 other seeds (the generators differ by
design, so only the means can agree; both turn a 32-bit output u into
(u >> 9) * 2^-23, so the sample distributions are identical by construction).
Interior gradients are deterministic and enter both sides unchanged.

Per gradient element: z = |mean_philox - mean_pcg| / sqrt(se_philox^2 + se_pcg^2),
se the standard error of each mean.  A boundary estimate is a sum of
heavy-tailed per-sample terms (colour jump / pdf), so 64-seed standard errors
are themselves noisy (PCG against PCG over disjoint seed sets shows the same
spread).  Bar: >= 97 % of the elements with spread within 3 sigma, none beyond
6 sigma, mean z^2 <= 2 (a systematic bias moves every element); elements without
spread (interior-only gradients) within 1e-4 of their array's scale.

CPU: the oracle's Philox against the oracle's PCG32 (64x64, 2x2 spp).
GPU: the CUDA path's Philox against the oracle's PCG32 on the 128x128, 4x4-spp
adjoint-verification scene with W*H boundary samples per run.
"""
import os

import numpy as np
import pytest

from dvg import BackwardOptions, RenderOptions, Rng, synth

SEEDS = 64
NAMES = ("d_points", "d_shape_stroke_width", "d_paint_params", "d_background")


def _setup(side, spp):
    import pyoracle

    sc = synth.adjoint_scene(0, side, side)
    opts = RenderOptions(samples_x=spp, samples_y=spp, seed=0, jitter=True, use_prefiltering=False)
    img = pyoracle.render(sc, opts)
    target = pyoracle.render(synth.adjoint_scene(1, side, side), opts)
    return sc, opts, (2.0 * (img - target)).astype(np.float32)


def _oracle_runs(sc, opts, dr, rng, base):
    import pyoracle

    nb = sc.width * sc.height
    threads = max(1, os.cpu_count() or 1)
    _, interior = pyoracle.render_backward(sc, opts, BackwardOptions(boundary_samples=nb), dr, passes=1,
                                           threads=threads)
    out = {n: [] for n in NAMES}
    for s in range(SEEDS):
        _, b = pyoracle.render_backward(sc, opts, BackwardOptions(rng=rng, boundary_seed=base + s, boundary_samples=nb),
                                        dr, passes=2, threads=threads)
        for n in NAMES:
            out[n].append(np.asarray(interior[n], np.float64) + np.asarray(b[n], np.float64))
    return out


def _compare(philox, pcg):
    zs = []
    for n in NAMES:
        a, o = np.stack(philox[n]), np.stack(pcg[n])
        ma, mo = a.mean(0), o.mean(0)
        se = np.sqrt(a.var(0, ddof=1) / len(a) + o.var(0, ddof=1) / len(o))
        scale = float(np.max(np.abs(mo))) + 1e-6
        flat = se <= 1e-7 * scale
        assert np.all(np.abs(ma - mo)[flat] <= 1e-4 * scale + 1e-6), n
        zs.append(np.abs(ma - mo)[~flat] / se[~flat])
    z = np.concatenate(zs)
    assert z.size > 50
    assert float(np.mean(z <= 3.0)) >= 0.97, f"{int(np.sum(z > 3.0))} of {z.size} beyond 3 sigma"
    assert float(np.max(z)) <= 6.0, f"max z {float(np.max(z)):.2f}"
    assert float(np.mean(z * z)) <= 2.0, f"mean z^2 {float(np.mean(z * z)):.2f}"


def test_oracle_philox_matches_pcg_in_expectation():
    sc, opts, dr = _setup(64, 2)
    _compare(_oracle_runs(sc, opts, dr, Rng.PHILOX, 1000), _oracle_runs(sc, opts, dr, Rng.PCG32, 5000))


@pytest.mark.gpu
def test_cuda_philox_matches_oracle_pcg_in_expectation():
    from dvg import Renderer

    sc, opts, dr = _setup(128, 4)
    nb = sc.width * sc.height
    r = Renderer(0)
    try:
        gpu = {n: [] for n in NAMES}
        for s in range(SEEDS):
            g = r.render_backward(sc, opts, BackwardOptions(rng=Rng.PHILOX, boundary_seed=1000 + s,
                                                            boundary_samples=nb), dr).buffers
            for n in NAMES:
                gpu[n].append(np.asarray(g[n], np.float64))
    finally:
        r.close()
    _compare(gpu, _oracle_runs(sc, opts, dr, Rng.PCG32, 5000))
