#!/usr/bin/env python
"""Benchmark of the render + backward hot path (one JSON line on rank 0).

A step is one forward render + L2 loss + backward (interior and boundary
passes) of one synthetic scene, through the library's fused device entry point
(dvg_fwd_bwd_l2_device) with the scene, the target and the gradients resident
in HBM.  Default workload: the 512x512, 4x4-spp mixed-primitive scene (256
shapes, Gaussian filter r=1, width*height boundary samples).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: forward+backward Msamples/s (pixel samples = W*H*spp per step) and
ms per step.  `e2e` repeats the step through the crate-shaped host calls
(dvg_render and dvg_render_backward with host scene description, host image
and host gradients; the L2 gradient is formed on the host in between).
Multi-GPU: one process per GPU, each rank renders its own scene (weak scaling,
no collective in the data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "diffvg-rs_b200"))

from dvg import BackwardOptions, Batch, DeviceGrads, Renderer, RenderOptions, synth  # noqa: E402
from dvg.abi import pack_scene as synth_pack  # noqa: E402
from dvg.shard import max_over_ranks, rank_seed, weak_scaling_rate  # noqa: E402

METRIC = "fwd+bwd Msamples/s (ms/iter), plain single-scene launch loop on one B200"
UNIT = "Msamples/s"
LARGE_FIT_LR = 0.1  # Adam step on path points (pixels) and paint parameters of the large fitting loop


def workload(name: str, seed: int):
    if name == "mixed":
        sc = synth.mixed_scene(seed)
        opts = synth.mixed_options()
        cfg = dict(workload="mixed-primitive scene 512x512, 4x4 spp, Gaussian r=1, 256 shapes "
                            "(128 cubic fills, 64 strokes, 32 circles, 32 ellipses), W*H boundary samples",
                   width=512, height=512, spp=16, shapes=256)
        target = synth.mixed_scene(seed + 1000)
        return sc, target, opts, BackwardOptions(boundary_samples=sc.width * sc.height), cfg
    if name == "plain":
        sc = synth.plain_scene(seed)
        opts = synth.plain_options()
        cfg = dict(workload="plain scene 256x256, 2x2 spp, box r=0.5, 16 closed cubic paths, target = the seed+1 "
                            "scene, W*H*spp boundary samples", width=256, height=256, spp=4, shapes=16)
        target = synth.plain_scene(seed + 1)
    elif name == "adjoint":
        sc = synth.adjoint_scene(seed)
        opts = synth.adjoint_options()
        cfg = dict(workload="adjoint-check scene 128x128, 4x4 spp, 4 filled cubic + 4 stroked quadratic paths, "
                            "W*H*spp boundary samples", width=128, height=128, spp=16, shapes=8)
        target = synth.adjoint_scene(seed + 1)
    elif name == "large":
        sc = synth.large_scene(seed)
        opts = RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=True, use_prefiltering=False)
        cfg = dict(workload="large scene 1024x1024, 4x4 spp, 4096 closed cubic paths x 16 segments, 25% stroked, "
                            "radial 3-stop fills, W*H*spp boundary samples", width=1024, height=1024, spp=16,
                   shapes=4096)
        target = synth.large_scene(seed + 7)
    else:
        raise SystemExit(f"unknown workload {name}")
    return sc, target, opts, BackwardOptions(), cfg


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def cpu_baseline(sc, opts, bopts, target_img, img, seconds: float, threads: int = 0):
    """CPU port of the crate's path (the oracle), bounded sample, `threads` host threads (0: all)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    threads = threads or os.cpu_count() or 1
    d_render = 2.0 * (img - target_img)
    total = sc.width * sc.height * opts.samples_x * opts.samples_y
    count = 4096
    n, setup, loop = pyoracle.fwd_bwd_sample(sc, opts, bopts, d_render, count, threads)
    # grow the sample until the loop takes a bounded ~`seconds` of host time
    if loop > 0:
        count = int(min(total, max(count, count * seconds / max(loop, 1e-6))))
        n, setup, loop = pyoracle.fwd_bwd_sample(sc, opts, bopts, d_render, count, threads)
    t = loop + setup * n / total  # per-call set-up amortised over the sample's share of the step
    return {"value": n / t / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} of {total} pixel samples spread evenly over the image (+ the same fraction of the "
                      f"{bopts.boundary_samples or total} boundary samples); set-up {setup:.2f}s amortised by that "
                      "fraction",
            "ms_per_step_extrapolated": t * total / n * 1e3}


def source_digest() -> str:
    """Digest of the library's kernel sources; ncu figures captured from other sources are stale."""
    h = hashlib.sha256()
    csrc = os.path.join(ROOT, "diffvg-rs_b200", "csrc")
    for n in sorted(os.listdir(csrc)):
        with open(os.path.join(csrc, n), "rb") as f:
            h.update(n.encode())
            h.update(f.read())
    return h.hexdigest()[:16]


def ncu_figures(workload: str):
    """Per-kernel ncu counters of one step of `workload` (profiles/ncu_step_<workload>.json, see
    ncu_import), whether they were captured from the current kernel sources, and the file."""
    path = os.path.join(ROOT, "profiles", f"ncu_step_{workload}.json")
    if not os.path.exists(path):
        return {}, False, None
    with open(path) as f:
        d = json.load(f)
    return d.get("kernels", {}), d.get("source_digest") == source_digest(), os.path.relpath(path, ROOT)


NCU_STEP_METRICS = ("gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum,"
                    "lts__t_sectors_op_red.sum,lts__t_sectors_op_atom.sum")


def ncu_import(csv_path: str, workload: str, digest: str = "") -> None:
    """Per-kernel sums over the launches of one captured step, keyed by kernel name, with the digest of
    the kernel sources they were captured from.  Capture (one GPU; warm-up outside the range):
      ncu --clock-control none --nvtx --nvtx-include dvg_step/ --metrics <NCU_STEP_METRICS> --csv
          --print-units base --log-file step.csv python bench.py --ncu-step --workload <w>"""
    import csv

    with open(csv_path) as f:
        rows = list(csv.DictReader(line for line in f if line.startswith('"')))
    names = {"gpu__time_duration.sum": "ns", "dram__bytes_read.sum": "dram_read", "dram__bytes_write.sum":
             "dram_write", "lts__t_sectors_op_red.sum": "red_sectors", "lts__t_sectors_op_atom.sum": "atom_sectors"}
    per = {}
    for row in rows:
        key = names.get(row["Metric Name"])
        if key is None:
            continue
        kname = row["Kernel Name"].replace("void ", "").split("(")[0].replace("dvgb::", "")
        per.setdefault(kname, {}).setdefault(row["ID"], {})[key] = float(row["Metric Value"].replace(",", ""))
    kernels = {}
    for kname, launches in per.items():
        s = {k: sum(l.get(k, 0.0) for l in launches.values()) for k in names.values()}
        kernels[kname] = {"launches": len(launches), "ms": s["ns"] / 1e6,
                          "dram_bytes": int(s["dram_read"] + s["dram_write"]),
                          "red_sectors": int(s["red_sectors"]), "atom_sectors": int(s["atom_sectors"])}
    out = {"workload": workload, "source_digest": digest or source_digest(),
           "what": "one fused step (forward + L2 + backward) captured by ncu after warm-up, L2 flushed before it; "
                   "per kernel, summed over its launches in the step; times are ncu's (serialised launches): "
                   "compare shares, not absolutes",
           "command": "ncu --clock-control none --nvtx --nvtx-include dvg_step/ --metrics " + NCU_STEP_METRICS +
                      " --csv --print-units base --log-file step.csv python bench.py --ncu-step --workload "
                      + workload + " --e2e-steps 0; python bench.py --ncu-import step.csv --workload " + workload,
           "kernels": dict(sorted(kernels.items(), key=lambda kv: -kv[1]["ms"]))}
    path = os.path.join(ROOT, "profiles", f"ncu_step_{workload}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(f"wrote {os.path.relpath(path, ROOT)}: {len(kernels)} kernels")


def compute_roofline(workload, prof, up, W, H, dev, clocks):
    """Compute roofline of the forward kernel: the crate's arithmetic for every test its BVH queries
    reach (profiles/roofline_work.json, counted by the oracle's counting build) over the kernel's
    average CUDA-event launch time, against the FP32 issue rate (SMs x 128 lanes x max SM clock, one
    unfused operation per lane per clock: the kernels are built without multiply-add contraction so
    that their decisions match the crate's).  The HBM figure is kept as a secondary field."""
    import torch

    with open(os.path.join(ROOT, "profiles", "roofline_work.json")) as f:
        work = json.load(f)["workloads"].get(workload)
    ms_tot, calls = prof.get("forward", (0.0, 1))
    avg_ms = ms_tot / max(calls, 1)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = clocks.get("sm_max_mhz") or 1965.0
    peak = sms * 128 * mhz * 1e6 / 1e12
    achieved = work["total_flops"] / (avg_ms / 1e3) / 1e12 if work and avg_ms > 0 else None
    kernels, fresh, src = ncu_figures(workload)
    # the forward kernel is a template over its resident CTAs per SM (k_forward<2>, k_forward<3>);
    # the captured step ran the shape the autotuner picked
    fk = next((v for k, v in kernels.items() if k == "k_forward" or k.startswith("k_forward<")), {})
    step_ms = sum(v[0] for v in prof.values())
    # HBM view of the same kernel: image-sized accumulators and weights, scene tables once
    npix = W * H
    scene_bytes = sum(a.nbytes for a in up.packed.arrays.values())
    alg_bytes = npix * (16 + 4) * 2 + scene_bytes
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak, hbm_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            hbm_peak, hbm_src = float(json.load(f).get("hbm_gbs", hbm_peak)), "measured"
    hbm_achieved = alg_bytes / (avg_ms / 1e3) / 1e9 if avg_ms > 0 else None
    return {
        "bound": "fp32_issue", "kernel": "k_forward", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
        "frac": achieved / peak if achieved is not None else None,
        "traffic": fk.get("dram_bytes") if fresh else None,
        "traffic_source": (f"{src}: ncu dram__bytes_read.sum + dram__bytes_write.sum of its one launch in a step"
                           if fresh and fk else "no ncu capture from the current kernel sources"),
        "peak_source": f"nominal: {sms} SMs x 128 FP32 lanes x {mhz:.0f} MHz (max SM clock sampled during the run)",
        "avg_launch_ms": avg_ms, "share_of_step": ms_tot / step_ms if step_ms else None,
        "work": {"flops_per_launch": work["total_flops"] if work else None,
                 "tests_per_launch": work["total_tests"] if work else None,
                 "source": "profiles/roofline_work.json (python oracle/count_work.py)"},
        "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s", "peak_source": hbm_src,
                "frac": hbm_achieved / hbm_peak if hbm_achieved else None, "algorithmic_bytes_per_launch": alg_bytes},
        "note": "the FP32 figure counts the crate's arithmetic per test (a libm call as one operation) and none of "
                "the per-sample jitter, transform, paint, compositing and splat work; the kernel skips tests the "
                "crate runs (exact culling), and it takes the crate's root decisions from f32 estimates polished "
                "by one f64 Newton step where bounds prove them equal (the crate's f64 formula otherwise)",
    }


def l2_atomic_probe(dev) -> float:
    """Measured rate of single-float atomic adds on this GPU: torch index_add_ of 2^26 values into 2^24
    floats at random int32 indices (one L2 reduction per value, plus the 8 bytes of index and value it
    reads), median of 5 timed runs, in G adds/s."""
    import torch

    n, m = 1 << 26, 1 << 24
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    idx = torch.randint(0, m, (n,), device=dev, dtype=torch.int32, generator=g)
    src = torch.ones(n, device=dev)
    dst = torch.zeros(m, device=dev)
    for _ in range(2):
        dst.index_add_(0, idx, src)
    ts = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.index_add_(0, idx, src)
        e1.record()
        torch.cuda.synchronize(dev)
        ts.append(e0.elapsed_time(e1))
    del idx, src, dst
    return n / (float(np.median(ts)) / 1e3) / 1e9


def l2_atomic_summary(workload, prof, dev):
    """L2 reduction sectors of one step (ncu, per kernel) against the measured atomic-add rate."""
    kernels, fresh, src = ncu_figures(workload)
    probe = l2_atomic_probe(dev)
    out = {"probe_gadds_per_s": probe,
           "probe": "torch index_add_ of 2^26 floats at random indices into 2^24 (one L2 reduction each)"}
    if not fresh:
        out["step"] = None
        out["note"] = "no ncu capture from the current kernel sources"
        return out
    step_ms = sum(v[0] for v in prof.values()) / 3.0
    per = {name: k.get("red_sectors", 0) + k.get("atom_sectors", 0) for name, k in kernels.items()}
    sectors = sum(per.values())
    rate = sectors / (step_ms / 1e3) / 1e9
    out["step"] = {"sectors": sectors, "gsectors_per_s_over_step": rate, "frac_of_probe": rate / probe,
                   "kernels": {k: v for k, v in per.items() if v > 0}, "source": src}
    return out


def large_fit(r, dev, lib_stream, steps, warmup, rank, lr=LARGE_FIT_LR):
    """Large fitting loop: 1024x1024, 4x4 spp, 4096 closed cubic paths of 16 segments
    (25 % stroked, radial 3-stop fills, group and shape transforms) fitted to the render
    of another seeded scene of the same structure; every iteration is one CUDA-graph
    replay of forward + L2 + backward + Adam (on path points and paint parameters) +
    on-device scene re-preparation, with no host work between iterations.  The loss of
    every 50th iteration is read back (a host synchronisation between two replays)."""
    import torch

    sc = synth.large_scene(rank_seed(0, rank))
    tgt_sc = synth.large_scene(rank_seed(1, rank) + 7)
    opts = RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=True, use_prefiltering=False)
    up = r.upload(sc)
    tu = r.upload(tgt_sc)
    batch = Batch(r, [up], opts, BackwardOptions())
    _, tgt, _ = batch.buffers(0)
    tu.render_device(opts, tgt.data_ptr())
    torch.cuda.synchronize(dev)
    tu.close()
    tuning = batch.autotune()
    batch.set_adam(lr, (0.9, 0.999), 1e-8, points=True, paints=True)
    batch.step(True)
    traj = [(1, float(batch.losses()[0]))]  # iteration 1: the loss of the initial scene
    for _ in range(warmup - 1):
        batch.step(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(lib_stream)
    for i in range(1, steps + 1):
        batch.step(True)
        if i % 50 == 0 or i == steps:
            traj.append((warmup + i, float(batch.losses()[0])))
    e1.record(lib_stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    samples = sc.width * sc.height * 16
    batch.close()
    up.close()
    return {"workload": "1024x1024, 4x4 spp, 4096 closed cubic paths x 16 segments, 25% stroked, radial 3-stop "
                        "fills, W*H*spp boundary samples, fitted to the render of another seeded scene; fwd + L2 + "
                        f"bwd + Adam (lr {lr}, points and paint parameters) + re-preparation per graph replay",
            "iterations": steps, "warmup": warmup, "ms_per_iter": ms, "msamples_per_s": samples / (ms / 1e3) / 1e6,
            "loss_first": traj[0][1], "loss_last": traj[-1][1], "loss_trajectory": traj,
            "launch_shape": {"sample_layout": tuning[0], "boundary_cell": tuning[1], "fragment_slots": tuning[2],
                             "work_queue": "persistent CTAs" if tuning[3] else "one CTA per item",
                             "forward_ctas_per_sm": 4 - tuning[4]}}


def prefiltered_step(r, dev, lib_stream, flush, steps, warmup, rank):
    """The crate's default mode: the mixed scene at 2x2 spp with prefiltering (smoothstep
    coverage from the signed distance, no boundary pass), one fused forward + L2 + backward
    per step, L2 flushed between steps, CUDA events on the library's stream."""
    import torch

    sc = synth.mixed_scene(rank_seed(0, rank))
    opts = RenderOptions(samples_x=2, samples_y=2, seed=0, jitter=True, use_prefiltering=True)
    bopts = BackwardOptions()
    up, tu = r.upload(sc), r.upload(synth.mixed_scene(rank_seed(0, rank) + 1000))
    n = sc.width * sc.height * 4
    tgt, img = torch.empty(n, device=dev), torch.empty(n, device=dev)
    loss = torch.zeros(1, device=dev)
    tu.render_device(opts, tgt.data_ptr())
    g = DeviceGrads(up.packed, dev)
    for _ in range(warmup):
        up.fwd_bwd_l2_device(opts, bopts, tgt.data_ptr(), img.data_ptr(), loss.data_ptr(), g)
    ts = []
    for _ in range(steps):
        with torch.cuda.stream(lib_stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        up.fwd_bwd_l2_device(opts, bopts, tgt.data_ptr(), img.data_ptr(), loss.data_ptr(), g)
        e1.record(lib_stream)
        torch.cuda.synchronize(dev)
        ts.append(e0.elapsed_time(e1))
    up.close()
    tu.close()
    ms = float(np.median(ts))
    samples = sc.width * sc.height * 4
    return {"workload": "mixed-primitive scene 512x512, 2x2 spp, prefiltered (the crate's default RenderOptions), "
                        "fwd + L2 + bwd", "steps": steps, "ms_per_step": ms, "msamples_per_s": samples / ms / 1e3}


def single_scene_sharded(r, dev, lib_stream, steps, warmup, rank, world):
    """One large scene split over all ranks (strong scaling): every rank renders a band
    of tiles and a range of boundary samples; NCCL sums the splat accumulators after the
    forward and the gradients after the backward (dvg.shard.SceneShardStep)."""
    import torch
    import torch.distributed as dist

    from dvg.shard import SceneShardStep

    sc = synth.large_scene(0)  # the same scene on every rank
    opts = RenderOptions(samples_x=4, samples_y=4, seed=0, jitter=True, use_prefiltering=False)
    bopts = BackwardOptions(boundary_samples=sc.width * sc.height)
    up = r.upload(sc)
    tu = r.upload(synth.large_scene(8))
    target = torch.empty(sc.width * sc.height * 4, device=dev)
    tu.render_device(opts, target.data_ptr())
    torch.cuda.synchronize(dev)
    tu.close()
    reduce = (lambda t: dist.all_reduce(t)) if world > 1 else (lambda t: None)
    step = SceneShardStep(up, opts, bopts, rank, world, reduce, device=dev)
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(lib_stream):
        for _ in range(warmup):
            step.step(target)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        for _ in range(steps):
            step.step(target)
        e1.record(lib_stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks([e0.elapsed_time(e1) / steps], dev)[0]
    up.close()
    samples = sc.width * sc.height * opts.samples_x * opts.samples_y
    return {"workload": "1024x1024, 4x4 spp, 4096 closed cubic paths x 16 segments (25% stroked), W*H boundary "
                        "samples, one scene split over the ranks (tile bands, boundary-sample ranges)",
            "world": world, "steps": steps, "ms_per_step": ms, "msamples_per_s": samples / (ms / 1e3) / 1e6,
            "scaling": "strong", "tiles_of_this_rank": list(step.tiles),
            "collectives": "NCCL all-reduce of the W*H*5 splat accumulators and of the gradient buffer per step"}


def batched_vs_plain(r, dev, lib_stream, flush, scenes, steps, label):
    """One batched CUDA-graph step over `scenes` against the loop of single-scene
    calls doing the same work (forward + L2 + backward, then the full optimisation
    step with Adam)."""
    import torch

    count = len(scenes)
    opts = synth.batched_options()
    bopts = BackwardOptions(boundary_samples=0)
    ups = [r.upload(s) for s in scenes]
    tgts = [r.upload(synth.plain_scene(1000 + i, s.width, s.height, 16)) for i, s in enumerate(scenes)]
    batch = Batch(r, ups, opts, bopts)
    plain = []
    for i, (up, tu) in enumerate(zip(ups, tgts)):
        _, tgt_b, _ = batch.buffers(i)
        tu.render_device(opts, tgt_b.data_ptr())
        n = up.scene.width * up.scene.height * 4
        plain.append((up, tgt_b, torch.empty(n, device=dev), torch.zeros(1, device=dev), DeviceGrads(up.packed, dev)))
    torch.cuda.synchronize(dev)

    def plain_step():
        for up, tgt, out, loss, g in plain:
            up.fwd_bwd_l2_device(opts, bopts, tgt.data_ptr(), out.data_ptr(), loss.data_ptr(), g)

    def timed(fn):
        fn()
        fn()
        torch.cuda.synchronize(dev)
        ms = []
        for _ in range(steps):
            with torch.cuda.stream(lib_stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(lib_stream)
            fn()
            e1.record(lib_stream)
            torch.cuda.synchronize(dev)
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    tuning = batch.autotune()
    t_plain = timed(plain_step)
    t_batch = timed(lambda: batch.step(True))
    # What batching can remove from the plain loop: the time its stream is not running a kernel
    # (launch latency and host work between the per-scene calls).  Kernel time from the library's
    # per-launcher CUDA events over one plain loop; launches per scene from its launch counter.
    torch.cuda.synchronize(dev)
    l0 = r.launch_count
    r.set_profiling(True)
    r.profile(reset=True)
    plain_step()
    prof = r.profile(reset=True)
    r.set_profiling(False)
    launches_per_scene = (r.launch_count - l0) / count
    kernel_ms = sum(v[0] for v in prof.values())
    gap_ms = max(t_plain - kernel_ms, 0.0)

    # Full optimisation step (forward, L2, backward, Adam lr 1e-2 on path points).
    # Batched: Adam and the scene re-preparation run on device inside the graph.
    # Plain: the crate's loop shape — per scene, host preparation + upload of the
    # current points, the fused device call, gradient read-back and a host Adam.
    batch.set_adam(1e-2, (0.9, 0.999), 1e-8, points=True)
    t_batch_opt = timed(lambda: batch.step(True))
    state = []
    for up in ups:
        pk = synth_pack(up.scene)
        n = pk.arrays["pts"].size
        state.append((up.scene, pk, np.zeros(n, np.float32), np.zeros(n, np.float32), [0]))

    def plain_opt_step():
        for k, (scene, pk, m, v, t) in enumerate(state):
            _, tgt_b, out_b, loss_b, g = plain[k][0], plain[k][1], plain[k][2], plain[k][3], plain[k][4]
            up = r.upload(scene, packed=pk)
            up.fwd_bwd_l2_device(opts, bopts, tgt_b.data_ptr(), out_b.data_ptr(), loss_b.data_ptr(), g)
            torch.cuda.synchronize(dev)
            grad = g.tensors["d_points"][: m.size].cpu().numpy()
            t[0] += 1
            m *= 0.9
            m += 0.1 * grad
            v *= 0.999
            v += 0.001 * grad * grad
            denom = np.sqrt(v) / np.sqrt(1.0 - 0.999 ** t[0]) + 1e-8
            pk.arrays["pts"] -= (1e-2 / (1.0 - 0.9 ** t[0])) * m / denom
            up.close()

    t_plain_opt = timed(plain_opt_step)
    samples = sum(s.width * s.height * 16 for s in scenes)
    out = {"scenes": count, "samples_per_step": samples,
           "batched_ms_per_step": t_batch, "plain_ms_per_step": t_plain,
           "scenes_per_s_batched_graph": count / (t_batch / 1e3), "scenes_per_s_plain_loop": count / (t_plain / 1e3),
           "msamples_per_s_batched": samples / (t_batch / 1e3) / 1e6, "speedup": t_plain / t_batch,
           "plain_loop_accounting": {
               "kernel_ms": kernel_ms, "not_in_a_kernel_ms": gap_ms, "launches_per_scene": launches_per_scene,
               "bound_from_gaps_only": t_plain / max(t_plain - gap_ms, 1e-9),
               "fill_gain_ms": kernel_ms - t_batch,
               "what": "kernel_ms: sum of the library's per-launcher CUDA-event times over one plain loop; "
                       "not_in_a_kernel_ms: the rest of the loop (launch latency, host work between calls). "
                       "Batching removes the second (bound_from_gaps_only = plain / kernel_ms, what removing "
                       "the gaps alone could give) and shortens the first by running many scenes' work items "
                       "in one grid instead of under-filled per-scene grids: fill_gain_ms = kernel_ms - "
                       "batched_ms_per_step (the graph replay has no host gaps), so plain - batched = "
                       "not_in_a_kernel_ms + fill_gain_ms"},
           "optimisation_step": {
               "batched_graph_ms": t_batch_opt, "plain_loop_ms": t_plain_opt,
               "scenes_per_s_batched_graph": count / (t_batch_opt / 1e3),
               "scenes_per_s_plain_loop": count / (t_plain_opt / 1e3), "speedup": t_plain_opt / t_batch_opt,
               "what": "fwd + L2 + bwd + Adam(lr 1e-2) on path points per scene; batched = one graph replay with "
                       "on-device Adam and scene re-preparation; plain = per scene host preparation + upload, "
                       "fused device call, gradient read-back, host Adam"},
           "workload": label, "launch_shape": {"sample_layout": tuning[0], "boundary_cell": tuning[1], "fragment_slots": tuning[2],
                             "work_queue": "persistent CTAs" if tuning[3] else "one CTA per item",
                             "forward_ctas_per_sm": 4 - tuning[4]}}
    batch.close()
    for u in ups + tgts:
        u.close()
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sc, target, opts, bopts, cfg = workload(args.workload, 0)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    # untimed inputs for the backward
    img = pyoracle.render_window(sc, opts, 0, 0, sc.width, sc.height, args.cpu_threads)
    tgt = pyoracle.render_window(target, opts, 0, 0, sc.width, sc.height, args.cpu_threads)
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(sc, opts, bopts, tgt, img, args.cpu_seconds / 4, args.cpu_threads)
    for _ in range(args.steps):
        vals.append(cpu_baseline(sc, opts, bopts, tgt, img, args.cpu_seconds / 2, args.cpu_threads))
    v = float(np.median([b["value"] for b in vals]))
    samples = cfg["width"] * cfg["height"] * cfg["spp"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": samples / (v * 1e6) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 root solves)",
            "data": "synthetic (seeded scene generator)", "config": cfg,
            "cpu_baseline": {**vals[-1], "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the crate's GPU path (CubeCL/wgpu) needs a graphics stack and is unavailable on this box; "
                    "its CPU path is timed through the C++ port (no Rust toolchain here)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-scenes", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=5)
    ap.add_argument("--large-fit-steps", type=int, default=200)
    ap.add_argument("--shard-steps", type=int, default=3)
    ap.add_argument("--prefilter-steps", type=int, default=5,
                    help="steps of the prefiltered leg (the crate's default mode; 0: skip)")
    ap.add_argument("--cpu-threads", type=int, default=0, help="host threads of the CPU baseline (0: all)")
    ap.add_argument("--ncu-step", action="store_true",
                    help="run the warm-up steps and one step inside the NVTX range dvg_step, then exit")
    ap.add_argument("--ncu-import", metavar="CSV",
                    help="turn an ncu --csv --print-units base capture of one --ncu-step step into "
                         "profiles/ncu_step_<workload>.json, then exit")
    ap.add_argument("--ncu-digest", default="",
                    help="kernel-source digest the --ncu-step run printed (default: the current sources')")
    args = ap.parse_args()
    if args.ncu_import:
        return ncu_import(args.ncu_import, args.workload, args.ncu_digest)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    sc, target_scene, opts, bopts, cfg = workload(args.workload, rank_seed(0, rank))
    W, H = sc.width, sc.height
    spp = opts.samples_x * opts.samples_y
    samples = W * H * spp
    r = Renderer(local)
    up = r.upload(sc)
    tgt_up = r.upload(target_scene)
    target = torch.empty(H * W * 4, device=dev)
    tgt_up.render_device(opts, target.data_ptr())
    out = torch.empty(H * W * 4, device=dev)
    loss = torch.zeros(1, device=dev)
    grads = DeviceGrads(up.packed, dev)
    lib_stream = torch.cuda.ExternalStream(r.stream_handle, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    tuning = up.autotune(opts, bopts, target.data_ptr())  # launch shape for this scene (dvg_scene_autotune)

    def step():
        up.fwd_bwd_l2_device(opts, bopts, target.data_ptr(), out.data_ptr(), loss.data_ptr(), grads)

    launches0 = r.launch_count
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    warm_launches = r.launch_count - launches0

    if args.ncu_step:
        # exactly one step inside the NVTX range "dvg_step" (L2 flushed before it), for an ncu capture
        # restricted to that range (ncu --nvtx --nvtx-include dvg_step/); no timing, no JSON line
        with torch.cuda.stream(lib_stream):
            flush.zero_()
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_push("dvg_step")
        step()
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_pop()
        print(f"ncu step of workload {args.workload}, kernel sources {source_digest()}", flush=True)
        up.close()
        tgt_up.close()
        r.close()
        return

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    evs = []
    launches_before = r.launch_count
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(lib_stream):
                flush.zero_()  # evict L2 between steps (outside the timed events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(lib_stream)
            step()
            e1.record(lib_stream)
            evs.append((e0, e1))
        torch.cuda.synchronize(dev)
    timed_launches = r.launch_count - launches_before
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = float(sum(step_ms))
    total_ms = max_over_ranks([total_ms], dev)[0]
    if world > 1:
        dist.barrier()
    value = weak_scaling_rate(args.steps * samples, world, total_ms) / 1e6

    # per-launcher device time (CUDA events inside the library), 3 extra untimed steps
    r.set_profiling(True)
    r.profile(reset=True)
    for _ in range(3):
        with torch.cuda.stream(lib_stream):
            flush.zero_()
        step()
    prof = r.profile(reset=True)
    r.set_profiling(False)
    torch.cuda.synchronize(dev)

    # end to end through the host API (scene description in, host image / host gradients out)
    e2e = None
    if args.e2e_steps > 0:
        tgt_host = target.view(H, W, 4).cpu().numpy()
        ts = []
        img_h = None
        # the L2 loss gradient, written in place every step, in page-locked memory
        d_render = torch.empty(tgt_host.shape, dtype=torch.float32, pin_memory=True).numpy()
        for i in range(args.e2e_steps + 1):
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(lib_stream)
            packed = synth_pack(sc)  # once per step: the scene may change between steps
            img_h = r.render(sc, opts, packed=packed).pixels
            np.subtract(img_h, tgt_host, out=d_render)
            d_render *= 2.0
            g = r.render_backward(sc, opts, bopts, d_render, packed=packed)
            e1.record(lib_stream)  # the calls block, so the events bracket host and device work
            torch.cuda.synchronize(dev)
            if i > 0:  # first call pays the one-time allocation of scratch buffers
                ts.append(e0.elapsed_time(e1) / 1e3)
        e2e_s = max_over_ranks([float(np.median(ts))], dev)[0]
        desc_bytes = sum(a.nbytes for a in up.packed.arrays.values())
        grad_bytes = int(g.buffers.flat().nbytes)
        e2e = {"value": samples * world / e2e_s / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(desc_bytes + d_render.nbytes),
               "d2h_bytes_per_step": int(img_h.nbytes + grad_bytes), "ms_per_step": e2e_s * 1e3,
               "path": "pack_scene + dvg_render + dvg_render_backward per step (host buffers: the image "
                       "and the loss gradient in page-locked memory; the backward reuses the scene, weights "
                       "and fragment codes dvg_render retained)"}

    fit = None
    if args.large_fit_steps > 0:
        fit = large_fit(r, dev, lib_stream, args.large_fit_steps, 3, rank)
        if world > 1:
            fit["ms_per_iter"] = max_over_ranks([fit["ms_per_iter"]], dev)[0]

    sharded = None
    if args.shard_steps > 0:
        sharded = single_scene_sharded(r, dev, lib_stream, args.shard_steps, 2, rank, world)

    prefiltered = None
    if args.prefilter_steps > 0:
        prefiltered = prefiltered_step(r, dev, lib_stream, flush, args.prefilter_steps, 3, rank)
        if world > 1:
            prefiltered["ms_per_step"] = max_over_ranks([prefiltered["ms_per_step"]], dev)[0]

    batched = None
    if args.batch_scenes > 0:
        batched = batched_vs_plain(
            r, dev, lib_stream, flush, synth.batched_scenes(seed=rank_seed(0, rank), count=args.batch_scenes),
            args.batch_steps, f"{args.batch_scenes} uneven scenes: side in {{128,256,512}}, log-uniform 4-1024 closed "
            "cubic paths (plain mix, paths shrink as sqrt(16/n)), 4x4 spp, box r=0.5, W*H*spp boundary samples")
        batched["small_scenes"] = batched_vs_plain(
            r, dev, lib_stream, flush, synth.small_scenes(seed=rank_seed(2, rank), count=256), args.batch_steps,
            "256 scenes of 64x64, 4-16 closed cubic paths (plain mix), 4x4 spp, box r=0.5, W*H*spp boundary samples")
        if world > 1:
            o = batched["optimisation_step"]
            mx = max_over_ranks([batched["batched_ms_per_step"], batched["plain_ms_per_step"],
                                 o["batched_graph_ms"], o["plain_loop_ms"]], dev)
            batched["batched_ms_per_step"], batched["plain_ms_per_step"] = mx[0], mx[1]
            o["batched_graph_ms"], o["plain_loop_ms"] = mx[2], mx[3]
            n = batched["scenes"] * world
            o["scenes_per_s_batched_graph"] = n / (mx[2] / 1e3)
            o["scenes_per_s_plain_loop"] = n / (mx[3] / 1e3)
            o["speedup"] = mx[3] / mx[2]
            sm = batched["small_scenes"]
            mx = max_over_ranks([sm["batched_ms_per_step"], sm["plain_ms_per_step"]], dev)
            sm["batched_ms_per_step"], sm["plain_ms_per_step"] = mx[0], mx[1]
            sm["speedup"] = mx[1] / mx[0]
            batched["scenes_per_s_batched_graph"] = n / (batched["batched_ms_per_step"] / 1e3)
            batched["scenes_per_s_plain_loop"] = n / (batched["plain_ms_per_step"] / 1e3)
            batched["speedup"] = batched["plain_ms_per_step"] / batched["batched_ms_per_step"]

    clock_summary = clocks.summary()
    roofline = compute_roofline(args.workload, prof, up, W, H, dev, clock_summary)
    roofline["l2_atomics"] = l2_atomic_summary(args.workload, prof, dev)
    prof_json = {k: {"ms_per_step": v[0] / 3.0, "calls_per_step": v[1] / 3.0} for k, v in prof.items()}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (f64 root solves, as the crate)",
        "data": "synthetic (seeded scene generator, no dataset)",
        "config": {**cfg, "boundary_samples": bopts.boundary_samples, "l2": "flushed between timed steps "
                   "(256 MiB write outside the timed events)", "parallelism": f"weak, {world} independent scene(s)",
                   "launch_shape": {"sample_layout": tuning[0], "boundary_cell": tuning[1],
                                    "fragment_slots": tuning[2], "forward_ctas_per_sm": 4 - tuning[4],
                                    "chosen_by": "dvg_scene_autotune"}},
        "roofline": roofline,
        "kernel_ms_per_step": prof_json,
        "gpu_launches": int(timed_launches), "clocks": clock_summary, "e2e": e2e,
        "batched_vs_plain": batched, "large_fit": fit, "single_scene_sharded": sharded,
        "prefiltered": prefiltered,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        img = out.view(H, W, 4).cpu().numpy()
        line["cpu_baseline"] = cpu_baseline(sc, opts, bopts, target.view(H, W, 4).cpu().numpy(), img,
                                            args.cpu_seconds, args.cpu_threads)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    up.close()
    tgt_up.close()
    r.close()


if __name__ == "__main__":
    main()
