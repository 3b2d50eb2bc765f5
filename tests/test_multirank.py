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
