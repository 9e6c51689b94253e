"""Benchmark of the MorseHGP3D product path on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the regular volumetric cloud, 37^3 = 50,653 lattice points jittered
by U[-0.25, 0.25] per axis, binary32 storage, seeded (synthetic; the
reference names no dataset).  K_max = 10.  A step is one pass of the product
path over one cloud; `config.stages` lists the stages inside the step:
canonical cloud + exact Morton LBVH, Boruvka EMST, compact k=1 forest, every
relevant pair and triple/quad critical-sphere support (rank <= 11), and the
direct Morse hierarchy (terminal facade, event journal, arm seeds, strict-arm
descent, frozen-root quotient, hyper-Kruskal forest journal for orders 1..10).

value : p95 over the K timed steps of the step time on the device timeline
        (CUDA events on the library's stream around the whole step; inputs
        already resident in HBM; the host-side forest sweep is inside).
e2e   : p95 over K steps of the same step through the public C ABI with host
        buffers (the reference's warm_e2e protocol): pinned host input copied
        in, and the hgp_reduced payload copied back to pinned host memory:
        EMST edges and exact lengths, k=1 forest arenas, the forest nodes (with
        the support of each node's level, which gives its exact level), child
        arena, forest batches and final roots of every order, and the vertical
        maps between adjacent orders; wall clock.
L2 is flushed (a 512 MiB write) before every timed step.

Multi-GPU: replicas only (one independent cloud per rank, different seeds),
barrier + max over ranks; no data-path collective.

--impl reference times the reference's own CPU code (oracle/_ref, compiled
from the reference sources) on rank 0 only, on the same cloud under a
work-unit budget: its exact pair stream resolves about 200 of the 1.28e9 pairs
per second, so the line reports the time-to-budget extrapolated to every pair
(a lower bound of its time for the workload) with the measured work units per
second and resolved fraction.

--chain WORKLOAD runs one pass of the chain on lattice:SIDE, uniform:N,
clustered:N or mixture:N and prints its stage times and work counters (the
harness of the profiles/ captures).
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

METRIC = "warm_e2e_p95_ms_50k_jittered_lattice_K10"
WORKLOAD = "jittered_lattice_37^3_f32"
K_MAX = 10
STAGES = ["canonical_cloud", "exact_morton_lbvh", "boruvka_emst", "k1_compact_forest", "pair_supports_rank_le_11",
          "higher_supports_rank_le_11", "direct_morse_hierarchy_orders_1_10",
          "vertical_maps_orders_2_10"]


def p95(xs):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), 95))


def spread(xs) -> dict:
    """p50 / p95 / p99 / max and the median absolute deviation of a list of times."""
    a = np.asarray(xs, dtype=np.float64)
    med = float(np.median(a))
    return {"p50": med, "p95": float(np.percentile(a, 95)), "p99": float(np.percentile(a, 99)),
            "max": float(a.max()), "mad": float(np.median(np.abs(a - med))), "n": int(len(a))}


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


def dist_setup():
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
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"  # gloo reduces host tensors
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---- the reference's own CPU code (budgeted protocol on the whole cloud) ---------------
# The reference's exact chain cannot finish this cloud: its pair stream resolves about 200
# pairs per second of the 1.28e9, so it is timed the way its own validation runs time it,
# under a work-unit budget on the whole cloud (morsehgp3d/docs/validation/phase9-pair-smoke-
# 2ed620b.json): canonical cloud + LBVH, then build_exact_pair_support_stream with
# maximum_work_unit_count = budget.  The time to resolve every pair is extrapolated linearly
# from the resolved fraction; it is a lower bound of the reference's time for the workload
# (the triple/quad stream and the hierarchy are not counted).  Its own full chain (pair and
# triple/quad streams, facade, journal, seeds, forest journal) is also timed on an 8-point
# corner of the cloud.
BUDGETS = (10_000, 100_000)
SAMPLE_SIDE = 2


def reference_sample(seed: int = 0) -> np.ndarray:
    import workloads
    return workloads.jittered_lattice(37, seed).reshape(37, 37, 37, 3)[:SAMPLE_SIDE, :SAMPLE_SIDE, :SAMPLE_SIDE] \
        .reshape(-1, 3).astype(np.float64)


def reference_step_seconds(pts: np.ndarray) -> dict:
    """Stage times of the reference chain on a small cloud (single thread, as the reference is)."""
    from oracle import pyoracle
    lb = pyoracle.lbvh_build(pts, "reference")["seconds"]
    pyoracle.emst_forest(pts, "reference")
    ef = pyoracle._text_call.seconds.copy()
    pyoracle.hierarchy(pts, K_MAX, "reference")
    hi = pyoracle._text_call.seconds.copy()
    return {"canonical_cloud": lb[0], "exact_morton_lbvh": lb[1], "boruvka_emst": ef[0],
            "k1_compact_forest": ef[1], "pair_and_higher_supports": hi[0], "direct_morse_hierarchy": hi[1]}


def reference_budgeted(pts: np.ndarray, budget: int) -> dict:
    """One budgeted run of the reference's pair stream on the whole cloud."""
    from oracle import pyoracle
    r = pyoracle.ref_pairs_budget(pts, K_MAX, budget)
    per_pair = r["stream_s"] / max(r["resolved_pairs"], 1)
    r["work_units_per_s"] = r["work_units"] / max(r["stream_s"], 1e-12)
    r["resolved_fraction"] = r["resolved_pairs"] / max(r["total_pairs"], 1)
    r["extrapolated_full_pair_stream_ms"] = 1e3 * (r["lbvh_s"] + per_pair * r["total_pairs"])
    return r


def reference_protocol_text() -> str:
    return ("reference CPU code (oracle/_ref, compiled from its sources), one thread: canonical cloud + LBVH + "
            "exact pair stream on the whole 50,653-point cloud under a work-unit budget; value = time-to-budget "
            "extrapolated to every pair by the resolved fraction (a lower bound of the full chain: the triple/"
            "quad stream and the hierarchy are not counted)")


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import pyoracle
    if not pyoracle.available("reference"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libehgp_ref.so was not built"}))
        return
    import workloads
    pts = workloads.jittered_lattice(37, 0).astype(np.float64)
    for _ in range(min(args.warmup, 1)):
        reference_budgeted(pts, BUDGETS[0])
    runs = [reference_budgeted(pts, BUDGETS[0]) for _ in range(max(1, min(args.steps, 10)))]
    vals = [r["extrapolated_full_pair_stream_ms"] for r in runs]
    v = p95(vals)
    sample = (f"{BUDGETS[0]} work units of the exact pair stream per step on the whole cloud "
              f"({runs[0]['resolved_pairs']} of {runs[0]['total_pairs']} pairs resolved, "
              f"{runs[0]['work_units_per_s']:.0f} work units/s), extrapolated")
    line = {"metric": METRIC, "value": v, "unit": "ms", "n_gpus": args.gpus, "steps": len(runs),
            "warmup": min(args.warmup, 1), "ms_per_step": float(np.mean(vals)), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "exact", "data": "synthetic", "impl": "reference",
            "value_kind": "extrapolated lower bound (pair stream only)",
            "config": {"workload": WORKLOAD, "points": int(len(pts)), "K_max": K_MAX, "stages": STAGES,
                       "protocol": reference_protocol_text(), "sample": sample},
            "measured": {"time_to_budget_s": [r["lbvh_s"] + r["stream_s"] for r in runs],
                         "work_units_per_s": float(np.median([r["work_units_per_s"] for r in runs])),
                         "resolved_fraction": runs[0]["resolved_fraction"]},
            "cpu_baseline": {"value": v, "unit": "ms", "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def cpu_baseline_line(ours_on_sample_ms: float | None) -> dict:
    from oracle import pyoracle
    if not pyoracle.available("reference"):
        return {"value": None, "unit": "ms", "cores": 1, "kind": "reference", "sample": "oracle/_ref not built"}
    import workloads
    pts = workloads.jittered_lattice(37, 0).astype(np.float64)
    budgeted = {str(b): reference_budgeted(pts, b) for b in BUDGETS}
    last = budgeted[str(BUDGETS[-1])]
    small = reference_sample(0)
    st = reference_step_seconds(small)
    return {"value": last["extrapolated_full_pair_stream_ms"], "unit": "ms", "cores": 1, "kind": "reference",
            "value_kind": "extrapolated lower bound (pair stream only)",
            "sample": (f"exact pair stream on the whole cloud at budgets {list(BUDGETS)} work units, extrapolated "
                       f"by the resolved fraction; full chain on an 8-point corner"),
            "protocol": reference_protocol_text(),
            "budgeted": budgeted,
            "full_chain_8_points": {"ms": 1e3 * sum(st.values()), "stage_ms": {k: 1e3 * v for k, v in st.items()},
                                    "gpu_same_sample_ms": ours_on_sample_ms},
            "host_cores_total": os.cpu_count()}


# ---- batched uneven clouds and a serving stream (one GPU) -------------------------------
BATCH_CLOUDS = 32          # clouds of the batched workload timed per run (of its 512)
SERVE_REQUESTS = 24        # requests of each serving-stream rate
WORKER_CHOICES = (1, 2, 4) # worker counts the batched runs compare; the best serves the stream


def _plain_payload(ctx, pts, K):
    """One cloud through the public API, one call at a time: host points in, the served
    payload (EMST edges, hierarchy arrays, node level supports) out."""
    ctx.lbvh_build(pts, outputs=False)
    return ctx.served_result(K)


def served_section(local: int) -> dict:
    """Batched uneven clouds (Gaussian mixtures of 1-6 components + 10 % noise, sizes
    log-uniform in [1,000, 20,000], binary32, K_max = 10): clouds/s of one cloud per call on
    one context against the serving engine with 1, 2 or 4 workers (the best is reported), all
    submitted at once.
    Serving stream: Poisson arrivals of clouds from the same generator with sizes log-uniform
    in [500, 20,000] and K_max uniform in {4, 10}, at rates relative to the served throughput;
    p50/p95/p99 latency (submit to result in host memory) and achieved clouds/s per rate."""
    import ehgp
    import workloads
    clouds = workloads.batched_uneven(BATCH_CLOUDS, seed=7)
    out = {"batched": {"workload": f"{BATCH_CLOUDS} of 512 mixture clouds, n log-uniform in [1000, 20000], f32",
                       "points": int(sum(len(c) for c in clouds))}}
    maxn = max(len(c) for c in clouds)
    # both paths are warmed on the largest clouds first, so that their buffers are sized
    # before the timed runs (device record buffers, hierarchy arenas, host arenas)
    largest = sorted(clouds, key=len)[-2:]
    with ehgp.Context(max_points=max(maxn, 20000), device=local) as ctx:
        for c in largest:
            _plain_payload(ctx, c, K_MAX)  # warm-up
        t0 = time.perf_counter()
        for c in clouds:
            _plain_payload(ctx, c, K_MAX)
        plain_s = time.perf_counter() - t0
    def served_rate(clouds_, workers):
        with ehgp.Server(workers=workers, max_points=20000, device=local) as srv:
            big = max(clouds_, key=len)
            for rid in [srv.submit(big, K_MAX) for _ in range(2 * workers)]:  # warm-up: every worker
                srv.wait(rid)
                srv.release(rid)
            t0 = time.perf_counter()
            ids = [srv.submit(c, K_MAX) for c in clouds_]
            bad = sum(srv.wait(r) != 0 for r in ids)
            wall = time.perf_counter() - t0
            for r in ids:
                srv.release(r)
        return len(clouds_) / wall, bad

    # the worker count is picked by measurement (each extra worker overlaps one cloud's host
    # forest pass with another's device stages, and costs host threads and device memory)
    per_w = {w: served_rate(clouds, w) for w in WORKER_CHOICES}
    best_w = max(per_w, key=lambda w: per_w[w][0])
    served_cps, bad = per_w[best_w]
    out["batched"].update({"plain_clouds_per_s": len(clouds) / plain_s, "served_clouds_per_s": served_cps,
                           "served_over_plain": served_cps * plain_s / len(clouds), "workers": best_w,
                           "served_clouds_per_s_by_workers": {str(w): v[0] for w, v in per_w.items()},
                           "failed": bad})
    # the same comparison on uniform clouds, whose step is dominated by the host forest pass
    ucl = [workloads.uniform_cube(int(n), 500 + i) for i, n in
           enumerate(np.exp(np.random.Generator(np.random.PCG64(5)).uniform(np.log(1000), np.log(20000), 32)))]
    with ehgp.Context(max_points=20000, device=local) as ctx:
        _plain_payload(ctx, max(ucl, key=len), K_MAX)
        t0 = time.perf_counter()
        for c in ucl:
            _plain_payload(ctx, c, K_MAX)
        uplain = time.perf_counter() - t0
    uper = {w: served_rate(ucl, w) for w in WORKER_CHOICES}
    ubest = max(uper, key=lambda w: uper[w][0])
    out["batched_uniform"] = {"workload": "32 uniform clouds, n log-uniform in [1000, 20000], f64",
                              "plain_clouds_per_s": len(ucl) / uplain, "served_clouds_per_s": uper[ubest][0],
                              "served_over_plain": uper[ubest][0] * uplain / len(ucl), "workers": ubest,
                              "served_clouds_per_s_by_workers": {str(w): v[0] for w, v in uper.items()},
                              "failed": uper[ubest][1]}
    with ehgp.Server(workers=best_w, max_points=20000, device=local) as srv:
        # serving stream at rates relative to the served throughput
        rng = np.random.Generator(np.random.PCG64(11))
        sizes = np.exp(rng.uniform(np.log(500), np.log(20000), SERVE_REQUESTS)).astype(int)
        reqs = [(workloads.mixture_cloud(int(n), rng), int(rng.choice([4, 10]))) for n in sizes]
        cap = served_cps
        rates = []
        for frac in (0.5, 1.0):
            lam = frac * cap
            gaps = rng.exponential(1.0 / lam, SERVE_REQUESTS)
            t0 = time.perf_counter()
            ids = []
            due = t0
            for (pts, K), g in zip(reqs, gaps):
                due += g
                while time.perf_counter() < due:
                    time.sleep(min(0.001, max(0.0, due - time.perf_counter())))
                ids.append(srv.submit(pts, K))
            fails = sum(srv.wait(r) != 0 for r in ids)
            wall = time.perf_counter() - t0
            lat = [srv.info(r)["latency_ms"] for r in ids]
            for r in ids:
                srv.release(r)
            rates.append({"offered_clouds_per_s": lam, "achieved_clouds_per_s": SERVE_REQUESTS / wall,
                          "latency_ms": spread(lat), "failed": fails})
        ok = [r for r in rates if r["latency_ms"]["p99"] < 100.0 and not r["failed"]]
        out["serving"] = {"workload": (f"{SERVE_REQUESTS} Poisson arrivals per rate, mixture clouds n log-uniform in "
                                       "[500, 20000], K_max in {4, 10}, f32"),
                          "workers": best_w, "rates": rates,
                          "clouds_per_s_at_p99_below_100ms": max((r["achieved_clouds_per_s"] for r in ok),
                                                                   default=None),
                          "server": srv.stats()}
    return out


# ---- our path ----------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import ctypes as C

    import torch

    import ehgp
    import workloads
    pts = workloads.jittered_lattice(37, rank)  # one independent cloud per rank (replicas)
    n = len(pts)
    ctx = ehgp.Context(max_points=n, device=local)
    pinned = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    pinned.copy_(torch.from_numpy(pts))
    host_pts = pinned.numpy()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    d_pts = torch.from_numpy(pts.astype(np.float64)).to(f"cuda:{local}")
    torch.cuda.synchronize(local)
    lib = ctx.lib
    m = n - 1
    forest = {"lv": np.empty((m, 4), np.uint64), "nodes": np.empty((m, 6), np.uint64),
              "child": np.empty(2 * m, np.uint64), "batches": np.empty((m, 7), np.uint64),
              "counts": np.zeros(4, np.uint64), "root": np.zeros(1, np.uint64)}
    fout = ehgp.K1ForestOut(*(forest[k].ctypes.data for k in ("lv", "nodes", "child", "batches", "counts", "root")))
    none_lbvh = ehgp.LbvhOut(None, None, None, None, None, None)
    cnt = np.zeros(1, np.uint64)
    hcnt = np.zeros(1, np.uint64)
    hc = ehgp.HierCounts()

    def pinned_np(count, dtype):
        nbytes = int(count) * np.dtype(dtype).itemsize
        t = torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)
        return t.numpy().view(dtype)[:count]

    def l2_flush():
        flush.fill_(1.0)
        torch.cuda.synchronize(local)

    def resident_step():
        """Device-resident step: supports stay in HBM; the hierarchy's host passes are inside."""
        ctx.step_begin()
        ctx._check(lib.ehgp_lbvh_build_device(ctx._h, C.c_void_p(d_pts.data_ptr()), n, C.byref(none_lbvh)))
        ctx._check(lib.ehgp_emst(ctx._h, None))
        ctx._check(lib.ehgp_k1_forest(ctx._h, C.byref(fout)))
        ctx._check(lib.ehgp_pairs(ctx._h, K_MAX, C.byref(ehgp.PairsOut(None, None, 0, cnt.ctypes.data))))
        ctx._check(lib.ehgp_higher(ctx._h, K_MAX, C.byref(ehgp.HigherOut(None, 0, hcnt.ctypes.data))))
        ctx._check(lib.ehgp_hierarchy(ctx._h, K_MAX, C.byref(hc)))
        return ctx.step_end()

    # one untimed pass sizes the host buffers of the e2e step
    resident_step()
    counts = {f: int(getattr(hc, f)) for f, _ in ehgp.HierCounts._fields_}
    e_u = pinned_np(m, np.uint32)
    e_v = pinned_np(m, np.uint32)
    e_D = pinned_np(m * 4, np.uint64).reshape(m, 4)
    rounds = np.zeros(1, np.uint32)
    eout = ehgp.EmstOut(e_u.ctypes.data, e_v.ctypes.data, e_D.ctypes.data, rounds.ctypes.data, None, 0, None)
    slack = 1.05
    f_nodes = pinned_np(int(counts["nodes"] * slack) + 64, ehgp.FOREST_NODE)
    f_child = pinned_np(int(counts["children"] * slack) + 64, np.uint32)
    f_batch = pinned_np(int(counts["journal_batches"] * slack) + 64, ehgp.FOREST_BATCH)
    f_root = pinned_np(64, ehgp.FOREST_ROOT)
    f_vert = pinned_np(int(counts["vertical_assignments"] * slack) + 64, ehgp.VERTICAL_ASSIGNMENT)
    hier_out = ehgp.HierOut(None, None, None, None, None, f_nodes.ctypes.data, f_child.ctypes.data, None, None,
                            None, None, f_batch.ctypes.data, f_root.ctypes.data, f_vert.ctypes.data)

    f_sup = pinned_np(5 * (int(counts["nodes"] * slack) + 64), np.uint32)

    def e2e_step():
        """The warm_e2e protocol: host points in; the hgp_reduced payload out into pinned host
        memory: the forests of orders 1..10 (nodes, child arena, batches, final roots) with the
        exact level of every node (the support of its level event), the vertical maps, and the
        EMST edges with their exact squared lengths and the compact k = 1 forest arenas.  The
        support records stay on the device (they are inputs of the hierarchy, not its payload)."""
        t0 = time.perf_counter()
        ctx.lbvh_build(host_pts, outputs=False)
        ctx._check(lib.ehgp_emst(ctx._h, C.byref(eout)))
        ctx._check(lib.ehgp_k1_forest(ctx._h, C.byref(fout)))
        ctx._check(lib.ehgp_hierarchy(ctx._h, K_MAX, C.byref(hc)))
        if (hc.nodes > len(f_nodes) or hc.children > len(f_child) or hc.journal_batches > len(f_batch)
                or hc.final_roots > len(f_root) or hc.vertical_assignments > len(f_vert)):
            raise RuntimeError("the hierarchy payload outgrew its host buffers")
        ctx._check(lib.ehgp_hier_copy(ctx._h, C.byref(hier_out)))
        lev = np.ascontiguousarray(f_nodes["level_event"][:hc.nodes])
        ctx._check(lib.ehgp_event_supports(ctx._h, lev.ctypes.data, hc.nodes, f_sup.ctypes.data))
        return 1e3 * (time.perf_counter() - t0)

    def payload_checksum():
        """64-bit checksums (xor and odd-weighted sum of the words) of the last e2e step's
        payload and its counts: the result must not change from step to step."""
        parts = [f_nodes[:hc.nodes], f_child[:hc.children], f_batch[:hc.journal_batches], f_root[:hc.final_roots],
                 f_vert[:hc.vertical_assignments], f_sup[:5 * hc.nodes], e_u, e_v, e_D,
                 np.array([getattr(hc, f) for f, _ in ehgp.HierCounts._fields_], np.uint64)]
        x = np.uint64(0)
        t = np.uint64(0)
        for a in parts:
            b = np.ascontiguousarray(a).reshape(-1).view(np.uint8)
            b = np.concatenate([b, np.zeros((-len(b)) % 8, np.uint8)]).view(np.uint64)
            x ^= np.bitwise_xor.reduce(b) if len(b) else np.uint64(0)
            with np.errstate(over="ignore"):
                t = t * np.uint64(0x9E3779B97F4A7C15) + (b * np.uint64(0xBF58476D1CE4E5B9)).sum(dtype=np.uint64)
        return f"{int(x):016x}{int(t):016x}"

    for _ in range(max(args.warmup, 3)):
        resident_step()
        e2e_step()
    check_first = payload_checksum()  # outside the timed steps
    barrier(world)
    dev_ms, e2e_ms, kern_ms = [], [], []
    hstats = None
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            l2_flush()
            dev_ms.append(resident_step())
            km, hstats = ctx.higher_stats()
            kern_ms.append(km)
        for _ in range(args.steps):
            l2_flush()
            e2e_ms.append(e2e_step())
    barrier(world)
    check_last = payload_checksum()
    value = max_over_ranks(p95(dev_ms), world)
    e2e = max_over_ranks(p95(e2e_ms), world)
    hs_last = ctx.hier_stats()
    if rank != 0:
        ctx.close()
        return
    # stage breakdown of one more step (device time per stage; host stages on the host clock)
    l2_flush()
    stage_ms = {}
    launches_per_step = 0
    ctx._check(lib.ehgp_lbvh_build_device(ctx._h, C.c_void_p(d_pts.data_ptr()), n, C.byref(none_lbvh)))
    stage_ms["lbvh"], l = ctx.last_timing()
    launches_per_step += l
    ctx._check(lib.ehgp_emst(ctx._h, None))
    stage_ms["emst"], l = ctx.last_timing()
    launches_per_step += l
    t0 = time.perf_counter()
    ctx._check(lib.ehgp_k1_forest(ctx._h, C.byref(fout)))
    stage_ms["k1_forest_host"] = 1e3 * (time.perf_counter() - t0)
    ctx._check(lib.ehgp_pairs(ctx._h, K_MAX, C.byref(ehgp.PairsOut(None, None, 0, cnt.ctypes.data))))
    stage_ms["pairs"], l = ctx.last_timing()
    launches_per_step += l
    ctx._check(lib.ehgp_higher(ctx._h, K_MAX, C.byref(ehgp.HigherOut(None, 0, hcnt.ctypes.data))))
    stage_ms["higher"], l = ctx.last_timing()
    launches_per_step += l
    t0 = time.perf_counter()
    ctx._check(lib.ehgp_hierarchy(ctx._h, K_MAX, C.byref(hc)))
    stage_ms["hierarchy_wall"] = 1e3 * (time.perf_counter() - t0)
    _, l = ctx.last_timing()
    launches_per_step += l
    hs = ctx.hier_stats()
    stage_ms["hierarchy_device"] = float(hs["device_ms"])
    stage_ms["hierarchy_descent"] = float(hs["descent_ms"])
    stage_ms["hierarchy_forest_host"] = float(hs["forest_ms"])
    launches = launches_per_step * args.steps
    # roofline of the dominant device kernel of the step (triple/quad enumeration, k_higher):
    # algorithmic bytes per launch from its counters: 28 B per candidate-set entry staged
    # (PointId + FP64 coordinates), 2568 B per point of per-cone radius table, 64 B per record.
    tested, classified, emitted, set_entries = (int(x) for x in hstats[:4])
    alg_bytes = 28 * set_entries + 2568 * n + 64 * emitted
    kmean = float(np.mean(kern_ms))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (kmean * 1e-3) / 1e9
    d2h = (e_u.nbytes + e_v.nbytes + e_D.nbytes + sum(forest[k].nbytes for k in forest)
           + int(hc.nodes) * (f_nodes.itemsize + 20) + int(hc.children) * 4
           + int(hc.journal_batches) * f_batch.itemsize + int(hc.final_roots) * f_root.itemsize
           + int(hc.vertical_assignments) * f_vert.itemsize)
    line = {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": float(np.mean(dev_ms)), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+exact", "data": "synthetic",
        "config": {"workload": WORKLOAD, "points": n, "K_max": K_MAX, "stages": STAGES, "seed": "rank",
                   "l2": "flushed 512MiB before each step", "parallelism": f"replicas{world}",
                   "pair_supports": int(cnt[0]), "higher_supports": int(hcnt[0]),
                   "hierarchy": {k: counts[k] for k in ("events", "journal_batches", "arm_seeds", "nodes",
                                                       "final_roots")},
                   "stage_ms": stage_ms},
        "latency_ms": {"device": spread(dev_ms), "e2e": spread(e2e_ms)},  # p50/p95/p99/max/MAD
        "payload_checksum": {"warmup": check_first, "last_step": check_last, "stable": check_first == check_last},
        "e2e": {"value": e2e, "unit": "ms", "h2d_bytes_per_step": int(pts.nbytes), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "gpu_launches_per_step": int(launches_per_step),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     # DRAM bytes of one k_higher launch: ncu capture of the 24^3 lattice (102.9 MB read +
                     # 1,755.9 MB written per launch over 13,824 owners at the 64-register budget),
                     # scaled per owner to this cloud
                     "traffic": (102938368 + 1755928576) * n / 13824,
                     "traffic_source": "ncu dram__bytes_read/write.sum on the 13,824-point case, scaled per owner",
                     "kernel": "k_higher (triple/quad support enumeration)",
                     "kernel_ms": kmean, "algorithmic_bytes": alg_bytes,
                     "work": {"status_tests": tested, "classified": classified, "records": emitted,
                              "candidate_set_entries": set_entries},
                     "note": "FP64 predicate-bound, not byte-bound; traffic is mostly local-memory spills",
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "clocks": clocks.summary(),
    }
    # roofline of the strict-arm descent step (k_arm_step), the largest share of the device
    # launch list: 40 B per facet (one descent step) + 32 B per LBVH node its ball query visits
    steps, visits = int(hs_last["descent_steps"]), int(hs_last["step_node_visits"])
    step_ms = float(hs_last["step_kernels_ms"])
    if step_ms > 0:
        d_bytes = 40 * steps + 32 * visits
        d_ach = d_bytes / (step_ms * 1e-3) / 1e9
        line["roofline_descent"] = {
            "bound": "hbm", "achieved": d_ach, "peak": hbm, "unit": "GB/s", "frac": d_ach / hbm, "traffic": None,
            "kernel": "k_arm_step (strict-arm descent step: exact facet miniball, ball query, exact top-k)",
            "kernel_ms_total": step_ms, "launches": int(hs_last["step_launches"]),
            "algorithmic_bytes": d_bytes, "work": {"descent_steps": steps, "node_visits": visits},
            "note": "FP64 miniball and exact top-k per thread; latency-bound, not byte-bound",
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    if world == 1 and not args.no_served:
        try:
            line.update(served_section(local))
        except Exception as exc:  # the headline line is printed either way
            line["served_error"] = f"{type(exc).__name__}: {exc}"
    if world == 1:
        # our own time on the reference's sample, for a like-for-like reading
        sample = reference_sample(0)
        with ehgp.Context(max_points=len(sample), device=local) as sctx:
            ts = []
            for _ in range(5):
                t0 = time.perf_counter()
                sctx.lbvh_build(sample, outputs=False)
                sctx.emst(with_minima=False)
                sctx.k1_forest()
                sctx.hierarchy(K_MAX, arrays=False)
                ts.append(1e3 * (time.perf_counter() - t0))
        line["cpu_baseline"] = cpu_baseline_line(float(np.median(ts)))
    print(json.dumps(line))
    ctx.close()


# ---- one pass of the chain on a named workload (stage times and work counters) ----------
def chain_workload(spec: str) -> tuple[str, np.ndarray]:
    """'lattice:SIDE[:SEED]' jittered unit lattice (binary32), 'uniform:N[:SEED]' U[0,1]^3,
    'clustered:N[:SEED]' the clustered near-degenerate generator (5 % snapped to 2^-10),
    'mixture:N[:SEED]' a Gaussian mixture with 10 % noise."""
    import workloads
    kind, *rest = spec.split(":")
    size = int(rest[0]) if rest else 24
    seed = int(rest[1]) if len(rest) > 1 else 0
    if kind == "lattice":
        return f"jittered_lattice_{size}^3_f32", workloads.jittered_lattice(size, seed)
    if kind == "uniform":
        return f"uniform_{size}", workloads.uniform_cube(size, seed)
    if kind == "clustered":
        return f"clustered_{size}", workloads.clustered(size, seed)
    if kind == "mixture":
        return f"mixture_{size}", workloads.mixture_cloud(size, np.random.Generator(np.random.PCG64(seed)))
    raise SystemExit(f"unknown workload {spec!r}")


def run_chain(spec: str, K: int, repeat: int) -> None:
    """Runs LBVH, EMST, k = 1 forest, pair and triple/quad supports and the hierarchy on one
    cloud `repeat` times and prints one JSON line per pass (stage times, counters)."""
    import ehgp
    name, pts = chain_workload(spec)
    n = len(pts)
    with ehgp.Context(max_points=n) as ctx:
        for r in range(repeat):
            out = {"workload": name, "points": n, "K": K, "pass": r}
            t0 = time.perf_counter()
            ctx.lbvh_build(pts, outputs=False)
            out["lbvh_ms"] = ctx.last_timing()[0]
            ctx.emst(with_minima=False)
            out["emst_ms"] = ctx.last_timing()[0]
            t = time.perf_counter()
            ctx.k1_forest()
            out["k1_forest_host_ms"] = 1e3 * (time.perf_counter() - t)
            cnt = np.zeros(1, np.uint64)
            import ctypes as C
            ctx._check(ctx.lib.ehgp_pairs(ctx._h, K, C.byref(ehgp.PairsOut(None, None, 0, cnt.ctypes.data))))
            out["pairs_ms"], out["pair_records"] = ctx.last_timing()[0], int(cnt[0])
            t = time.perf_counter()
            ctx._check(ctx.lib.ehgp_higher(ctx._h, K, C.byref(ehgp.HigherOut(None, 0, cnt.ctypes.data))))
            out["higher_wall_ms"] = 1e3 * (time.perf_counter() - t)
            out["higher_ms"] = ctx.last_timing()[0]
            km, st = ctx.higher_stats()
            out["higher_records"] = int(cnt[0])
            out["k_higher_ms"] = km
            out["higher_counters"] = [int(x) for x in st]
            t = time.perf_counter()
            try:
                ctx.hierarchy(K, arrays=False)
                out["decision"] = "complete"
            except ehgp.DegenerateError:
                out["decision"] = "refused: relevant extra-shell diagnostics"
            out["hierarchy_wall_ms"] = 1e3 * (time.perf_counter() - t)
            hs = ctx.hier_stats()
            out["hierarchy"] = {k: hs[k] for k in ("device_ms", "descent_ms", "forest_ms", "slowest_order_ms",
                                                   "host_orders_ms", "host_offsets_ms", "host_vertical_ms",
                                                   "order_ms", "arms", "events")}
            out["hierarchy_counts"] = ctx.last_hier_counts
            out["total_wall_ms"] = 1e3 * (time.perf_counter() - t0)
            print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chain", default=None, metavar="WORKLOAD",
                    help="one pass of the chain on lattice:SIDE, uniform:N, clustered:N or mixture:N (stage times)")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--no-served", action="store_true", help="skip the batched and serving measurements")
    ap.add_argument("--K", type=int, default=K_MAX)
    args = ap.parse_args()
    if args.chain:
        run_chain(args.chain, args.K, args.repeat)
        return
    if args.impl == "reference":
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup()
    run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
