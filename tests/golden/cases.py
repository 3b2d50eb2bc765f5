"""Golden cases: each names a seeded scene, its options and what is recorded.

Shared by make_golden.py (writes golden.npz from the oracle) and the tests that
read the fixtures back (oracle on the CPU, the CUDA path on the GPU).
"""
from __future__ import annotations

import numpy as np

from dvg import BackwardOptions, RenderOptions, Rng, synth


def _plain_opts():
    return synth.plain_options()


CASES = {
    # name: (scene factory, render options, backward options or None for render-only)
    "plain64_render": (lambda: synth.plain_scene(0, 64, 64, 8), _plain_opts, None),
    "mixed128_render": (lambda: synth.mixed_scene(3, 128, 128, scale=0.125, size_scale=0.25), synth.mixed_options,
                        None),
    "primitives_render": (synth.primitives_scene,
                          lambda: RenderOptions(samples_x=4, samples_y=4, seed=3, jitter=True, use_prefiltering=False),
                          None),
    "primitives_prefilter_render": (synth.primitives_scene,
                                    lambda: RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=True,
                                                          use_prefiltering=True), None),
    "plain48_backward": (lambda: synth.plain_scene(0, 48, 48, 6), _plain_opts, lambda: BackwardOptions()),
    "primitives_backward": (synth.primitives_scene,
                            lambda: RenderOptions(samples_x=2, samples_y=2, seed=5, jitter=True,
                                                  use_prefiltering=False),
                            lambda: BackwardOptions(compute_translation=True)),
    "primitives_prefilter_backward": (synth.primitives_scene,
                                      lambda: RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=True,
                                                            use_prefiltering=True),
                                      lambda: BackwardOptions(compute_translation=True)),
    "plain40_philox_backward": (lambda: synth.plain_scene(3, 40, 40, 5), _plain_opts,
                                lambda: BackwardOptions(rng=Rng.PHILOX, boundary_seed=1234, boundary_samples=5000)),
}


def d_render_for(image: np.ndarray) -> np.ndarray:
    """Seeded L2 adjoint: 2 * (image - clip(image + N(0, 0.1)))."""
    rng = np.random.default_rng(11)
    target = np.clip(image + rng.normal(0, 0.1, image.shape).astype(np.float32), 0, 1)
    return (2.0 * (image - target)).astype(np.float32)


def build(name: str):
    scene_fn, opts_fn, bopts_fn = CASES[name]
    return scene_fn(), opts_fn(), (bopts_fn() if bopts_fn else None)
