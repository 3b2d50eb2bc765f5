"""Linear BVH (Morton codes, key sort, Karras topology, bottom-up bounds).

CPU: the oracle's twin builds a valid tree (every node reached once, keys sorted
and unique, every parent box the union of its children's, leaves = the input boxes).
GPU: dvg_lbvh_build gives the same keys, topology and bounds bit for bit, including
boxes with identical centres (equal Morton codes, ordered by index) and n = 1, 2, 3.
"""
import numpy as np
import pytest


def _boxes(n, seed, clustered=False):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-50.0, 900.0, (n, 2))
    if clustered:
        c[: n // 2] = c[0]  # half the boxes share one centre
    h = rng.uniform(0.0, 20.0, (n, 2))
    return np.concatenate([c - h, c + h], 1).astype(np.float32)


CASES = [(1, 0, False), (2, 1, False), (3, 2, False), (17, 3, False), (1000, 4, False), (4096, 5, True),
         (20000, 6, False)]


def _check_tree(boxes, keys, ch, bounds):
    n = boxes.shape[0]
    assert n == 1 or all(int(keys[i]) < int(keys[i + 1]) for i in range(n - 1))
    assert sorted(int(k) & 0xFFFFFFFF for k in keys) == list(range(n))
    for k in range(n):
        assert np.array_equal(bounds[n - 1 + k], boxes[int(keys[k]) & 0xFFFFFFFF])
    seen = np.zeros(2 * n - 1, np.int64)
    stack = [0]
    while stack:
        v = stack.pop()
        seen[v] += 1
        if v < n - 1:
            a, b = ch[v]
            stack += [int(a), int(b)]
            u = np.concatenate([np.minimum(bounds[a, :2], bounds[b, :2]), np.maximum(bounds[a, 2:], bounds[b, 2:])])
            assert np.array_equal(bounds[v], u)
    assert np.all(seen == 1)


@pytest.mark.parametrize("n,seed,clustered", CASES[:6])
def test_cpu_twin_builds_a_valid_tree(n, seed, clustered):
    import pyoracle

    b = _boxes(n, seed, clustered)
    _check_tree(b, *pyoracle.lbvh_build(b))


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed,clustered", CASES)
def test_gpu_lbvh_matches_cpu_twin(n, seed, clustered):
    import pyoracle
    from dvg import Renderer

    b = _boxes(n, seed, clustered)
    r = Renderer(0)
    try:
        kg, cg, bg = r.lbvh_build(b)
    finally:
        r.close()
    kc, cc, bc = pyoracle.lbvh_build(b)
    assert np.array_equal(kg, kc)
    assert np.array_equal(cg, cc)
    assert np.array_equal(bg, bc)
