"""The multi-GPU plumbing on CPU: two gloo ranks (127.0.0.1) run the same shard /
seed / max-over-ranks logic bench.py runs over NCCL, plus each rank packs its own
scenes (weak scaling: disjoint seeds, no data-path exchange)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from dvg import synth
        from dvg.abi import pack_scene
        from dvg.shard import max_over_ranks, rank_seed, shard_range, weak_scaling_rate

        b, e = shard_range(64, rank, world)
        seed = rank_seed(0, rank)
        scenes = synth.batched_scenes(seed=seed, count=4)
        digest = [float(pack_scene(s).arrays["pts"].sum()) for s in scenes]
        ms = 10.0 + 5.0 * rank  # stand-in per-rank step times
        mx = max_over_ranks([ms, -ms])
        out.put((rank, b, e, seed, digest, mx, weak_scaling_rate(100.0, world, mx[0])))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, WORLD, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(WORLD))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, b0, e0, s0, d0, m0, v0), (r1, b1, e1, s1, d1, m1, v1) = res
    assert (b0, e0, b1, e1) == (0, 32, 32, 64)  # disjoint cover of the units
    assert s0 != s1 and d0 != d1  # each rank owns different scenes
    assert m0 == m1 == [15.0, -10.0]  # max over ranks, identical on every rank
    assert v0 == v1 == pytest.approx(100.0 * 2 / 0.015)


def test_shard_range_covers_everything():
    from dvg.shard import shard_range

    for n in (0, 1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            assert max(e - b for b, e in spans) - min(e - b for b, e in spans) <= 1


def test_cost_range_covers_everything_and_balances():
    import numpy as np

    from dvg.shard import cost_range, shard_range

    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 64, 257):
        for world in (1, 2, 3, 8):
            for costs in (rng.integers(1, 50, n), rng.pareto(1.5, n) + 1.0, np.zeros(n), np.ones(n)):
                spans = [cost_range(list(costs), r, world) for r in range(world)]
                assert spans[0][0] == 0 and spans[-1][1] == n
                assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
                assert all(b <= e for b, e in spans)
                total = float(np.sum(costs))
                if total > 0:
                    # every rank's cost is within one unit's cost of an equal share
                    for b, e in spans:
                        assert abs(float(np.sum(costs[b:e])) - total / world) <= float(np.max(costs)) + 1e-9
                else:
                    assert spans == [shard_range(n, r, world) for r in range(world)]


class _FakeShardScene:
    """Stands in for an uploaded scene on CPU: each shard call writes a value that
    names the rank into the buffers it is handed, so the test sees what the step
    summed across ranks and in which order the calls came."""

    def __init__(self, scene, packed, rank, calls):
        self.scene, self.packed, self.rank, self.calls = scene, packed, rank, calls
        self.renderer = self

    @staticmethod
    def _view(ptr, n):
        import ctypes

        import numpy as np

        return np.ctypeslib.as_array((ctypes.c_float * n).from_address(ptr))

    def tile_count(self):
        return 7

    def tile_groups(self):  # uneven work: the first tile holds most of the groups
        return [9, 0, 0, 1, 1, 1, 2]

    def shard_forward(self, options, tiles, accum_ptr, wsum_ptr):
        n = self.scene.width * self.scene.height
        self.calls.append(("forward", tuple(tiles)))
        self._view(accum_ptr, 4 * n)[:] = 1.0 + self.rank
        self._view(wsum_ptr, n)[:] = 10.0 * (1 + self.rank)

    def shard_resolve(self, accum_ptr, wsum_ptr, out_ptr):
        n = self.scene.width * self.scene.height
        self.calls.append(("resolve", float(self._view(accum_ptr, 1)[0]), float(self._view(wsum_ptr, 1)[0])))
        self._view(out_ptr, 4 * n)[:] = self._view(accum_ptr, 4 * n)

    def l2_device(self, image_ptr, target_ptr, n, d_render_ptr, loss_ptr):
        self.calls.append(("l2", n))

    def shard_backward(self, options, bopts, tiles, samples, d_render_ptr, wsum_ptr, grads):
        self.calls.append(("backward", tuple(tiles), tuple(samples)))
        grads.tensors["d_points"][:] = 100.0 * (1 + self.rank)


def _shard_worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from dvg import BackwardOptions, RenderOptions, synth
        from dvg.abi import pack_scene
        from dvg.shard import SceneShardStep

        sc = synth.plain_scene(3, 32, 16, 3)
        calls = []
        fake = _FakeShardScene(sc, pack_scene(sc), rank, calls)
        opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=True, use_prefiltering=False)
        step = SceneShardStep(fake, opts, BackwardOptions(boundary_samples=1001), rank, world, dist.all_reduce,
                              device="cpu")
        step.step(torch.zeros(32 * 16 * 4))
        out.put((rank, calls, float(step.grads.tensors["d_points"][0]), float(step.image[0])))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_single_scene_split_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, WORLD, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(WORLD))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, c0, g0, i0), (r1, c1, g1, i1) = res
    # tiles split by cost (groups + 1 = 10,1,1,2,2,2,3: half of 21 falls in tile 1) -> [0, 1) + [1, 7);
    # boundary samples 1001 -> [0, 501) + [501, 1001)
    assert c0[0] == ("forward", (0, 1)) and c1[0] == ("forward", (1, 7))
    assert c0[-1] == ("backward", (0, 1), (0, 501)) and c1[-1] == ("backward", (1, 7), (501, 1001))
    # the accumulators were summed before the resolve, the gradients after the backward
    assert c0[1] == c1[1] == ("resolve", 3.0, 30.0)
    assert [c[0] for c in c0] == ["forward", "resolve", "l2", "backward"]
    assert g0 == g1 == 300.0 and i0 == i1 == 3.0
