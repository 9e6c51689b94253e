"""Benchmark of the MorseHGP3D product path on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the regular volumetric cloud, 37^3 = 50,653 lattice points jittered
by U[-0.25, 0.25] per axis, binary32 storage, seeded (no dataset involved).
A step is one pass of the device pipeline over one cloud.  The stages that
exist so far run inside the step; `config.stages` names them.

value  : p95 over the K timed steps of the device time of one step (CUDA events
         on the library's stream, inputs already resident in HBM), max over ranks.
e2e    : p95 over K steps of the same work through the public C ABI with host
         buffers: pinned host->device copy of the points, the build, and the
         device->host copy of the full reference-layout result, wall clock.
L2 is flushed (a 512 MiB write) before every timed step.

Multi-GPU: replicas only (one independent cloud per rank, different seeds),
barrier + max over ranks; no data-path collective.

--impl reference times the reference's own CPU code of the same stages
(oracle/_ref, compiled from the reference sources), on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "e-hgp_b200")]

METRIC = "warm_e2e_p95_ms_50k_jittered_lattice"
WORKLOAD = "jittered_lattice_37^3_f32"
STAGES = ["canonical_cloud", "exact_morton_lbvh"]
BYTES_PER_POINT_LBVH = 310  # algorithmic bytes per point of the Morton/LBVH build


def p95(xs):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), 95))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows: list[list[str]] = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 2 + i and r[2 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_reference_time(pts64: np.ndarray, budget_s: float = 10.0, max_reps: int = 20) -> dict:
    """The reference's own CPU code (oracle/_ref) on the same cloud, 1 thread."""
    from oracle import pyoracle
    if not pyoracle.available("reference"):
        return {"value": None, "unit": "ms", "cores": 1, "kind": "reference", "sample": "oracle/_ref not built"}
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < max_reps and (not times or time.perf_counter() < t_end):
        r = pyoracle.lbvh_build(pts64, "reference")
        times.append(1e3 * float(r["seconds"].sum()))
    return {"value": p95(times), "unit": "ms", "cores": 1, "kind": "reference",
            "sample": f"full {len(pts64)}-point cloud, {len(times)} reps, p95; "
                      f"CanonicalPointCloud::rejecting_duplicates + MortonLbvhIndex::build, single thread",
            "host_cores_total": os.cpu_count()}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import workloads
    pts = workloads.jittered_lattice(37, 0).astype(np.float64)
    from oracle import pyoracle
    if not pyoracle.available("reference"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libehgp_ref.so was not built"}))
        return
    for _ in range(args.warmup):
        pyoracle.lbvh_build(pts, "reference")
    times = []
    for _ in range(args.steps):
        r = pyoracle.lbvh_build(pts, "reference")
        times.append(1e3 * float(r["seconds"].sum()))
    v = p95(times)
    line = {"metric": METRIC, "value": v, "unit": "ms", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(times)), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "exact", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "points": int(len(pts)), "stages": STAGES, "seed": 0},
            "cpu_baseline": {"value": v, "unit": "ms", "cores": 1, "kind": "reference",
                             "sample": f"full cloud, {args.steps} steps, single thread (reference CPU code is single-threaded)"},
            "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_ours(args, world, rank, local):
    import torch

    import ehgp
    import workloads
    pts = workloads.jittered_lattice(37, rank)  # one independent cloud per rank (replicas)
    n = len(pts)
    ctx = ehgp.Context(max_points=n, device=local)
    # pinned host copy of the input and host result buffers for the e2e leg
    pinned = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    pinned.copy_(torch.from_numpy(pts))
    host_pts = pinned.numpy()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def l2_flush():
        flush.fill_(1.0)
        torch.cuda.synchronize(local)

    # device-resident leg: inputs already in HBM (widened binary64 on device)
    d_pts = torch.from_numpy(pts.astype(np.float64)).to(f"cuda:{local}")
    torch.cuda.synchronize(local)
    import ctypes as C
    out_none = ehgp.LbvhOut(None, None, None, None, None, None)

    def device_step():
        st = ctx.lib.ehgp_lbvh_build_device(ctx._h, C.c_void_p(d_pts.data_ptr()), n, C.byref(out_none))
        ctx._check(st)
        return ctx.last_timing()

    for _ in range(max(args.warmup, 3)):
        device_step()
        ctx.lbvh_build(host_pts)
    barrier(world)
    dev_ms, e2e_ms, launches = [], [], 0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            l2_flush()
            ms, nl = device_step()
            dev_ms.append(ms)
            launches += nl
        for _ in range(args.steps):
            l2_flush()
            t0 = time.perf_counter()
            snap = ctx.lbvh_build(host_pts)
            e2e_ms.append(1e3 * (time.perf_counter() - t0))
            launches += ctx.last_timing()[1]
    barrier(world)
    value = max_over_ranks(p95(dev_ms), world)
    e2e = max_over_ranks(p95(e2e_ms), world)
    if rank != 0:
        ctx.close()
        return
    d2h = snap.leaves.nbytes + snap.nodes.nbytes + snap.source_index.nbytes + 5 * 8 + 6 * 8 + 8
    alg_bytes = BYTES_PER_POINT_LBVH * n
    mean_ms = float(np.mean(dev_ms))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (mean_ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+exact", "data": "synthetic",
        "config": {"workload": WORKLOAD, "points": n, "stages": STAGES, "seed": "rank", "l2": "flushed 512MiB",
                   "parallelism": f"replicas{world}"},
        "e2e": {"value": e2e, "unit": "ms", "h2d_bytes_per_step": int(pts.nbytes), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "kernel": "whole LBVH build (all stages)",
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "clocks": clocks.summary(),
    }
    if world == 1:
        line["cpu_baseline"] = cpu_reference_time(pts.astype(np.float64))
    print(json.dumps(line))
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    world, rank, local = dist_setup(args) if args.impl == "ours" else (
        int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
