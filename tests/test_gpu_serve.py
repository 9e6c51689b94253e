"""Serving engine (include/ehgp.h ehgp_server_*): continuous batching of many clouds.

* Each cloud's served result (forest nodes with the supports of their levels, child arena,
  forest batches, final roots, vertical maps, EMST edges) equals, array for array, the
  result of the same cloud run alone on a context of its own - with all clouds submitted at
  once, and with clouds arriving while others run.
* Admission by device memory: with a budget that holds one request at a time, requests
  wait for memory and still complete with the same results.
* Refusals: a cloud above max_points, K outside 1..10.
"""
import time

import numpy as np
import pytest

import ehgp
import workloads

pytestmark = pytest.mark.gpu

KEYS = ("nodes", "children", "batches", "roots", "vertical", "node_supports", "emst_u", "emst_v")


def _clouds(count=16, seed=3):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(300), np.log(3000))))
        pts = workloads.mixture_cloud(n, rng) if i % 3 else workloads.uniform_cube(n, 100 + i)
        out.append((pts, 4 if i % 2 else 10))
    return out


@pytest.fixture(scope="module")
def alone():
    """Every cloud run alone on one context (the plain path)."""
    clouds = _clouds()
    res = []
    with ehgp.Context(max_points=4096) as ctx:
        for pts, K in clouds:
            ctx.lbvh_build(pts, outputs=False)
            res.append({k: np.array(v, copy=True) for k, v in ctx.served_result(K).items()})
    return clouds, res


def _same(a, b):
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k


def test_gpu_served_equals_alone_all_at_once(alone):
    clouds, want = alone
    with ehgp.Server(workers=4, max_points=4096) as srv:
        ids = [srv.submit(p, K) for p, K in clouds]
        for i, rid in enumerate(ids):
            assert srv.wait(rid) == 0, srv.info(rid)["error"]
            _same(srv.result(rid), want[i])
            srv.release(rid)
        st = srv.stats()
        assert st["completed"] == len(clouds) and st["queued"] == 0 and st["running"] == 0


def test_gpu_served_equals_alone_with_arrivals(alone):
    """Clouds arrive while others run: each is admitted as a worker frees up."""
    clouds, want = alone
    with ehgp.Server(workers=3, max_points=4096) as srv:
        ids = []
        for i, (p, K) in enumerate(clouds):
            ids.append(srv.submit(p, K))
            if i % 4 == 3:
                time.sleep(0.02)
        running_seen = False
        for i, rid in enumerate(ids):
            running_seen |= srv.poll(ids[-1]) in (ehgp.REQ_QUEUED, ehgp.REQ_RUNNING)
            assert srv.wait(rid) == 0
            _same(srv.result(rid), want[i])
        infos = [srv.info(r) for r in ids]
        assert len({i["worker"] for i in infos}) == 3
        assert all(i["latency_ms"] >= i["service_ms"] > 0 for i in infos)


def test_gpu_server_admission_waits_for_memory(alone):
    """Six copies of the largest cloud on four workers with a budget that holds one
    request's reservation (its estimate before any measurement: 120 KiB per point + 64 MiB)
    and not two: the requests run one at a time, waiting for memory, with the same results."""
    import torch
    clouds, want = alone
    big = max(range(len(clouds)), key=lambda i: len(clouds[i][0]))
    pts, K = clouds[big]
    est = 120 * 1024 * len(pts) + (64 << 20)
    total = torch.cuda.get_device_properties(0).total_memory
    with ehgp.Server(workers=4, max_points=4096, hbm_fraction=1.5 * est / total) as srv:
        ids = [srv.submit(pts, K) for _ in range(6)]
        for rid in ids:
            assert srv.wait(rid) == 0
            _same(srv.result(rid), want[big])
        infos = [srv.info(r) for r in ids]
        assert srv.stats()["memory_waits"] > 0
        # one at a time: no two service intervals overlap
        spans = sorted((i["queued_ms"], i["queued_ms"] + i["service_ms"]) for i in infos)
        assert all(b[0] >= a[1] - 1.0 for a, b in zip(spans, spans[1:]))


def test_gpu_server_refusals():
    with ehgp.Server(workers=1, max_points=1000) as srv:
        with pytest.raises(ehgp.CapacityError):
            srv.submit(workloads.uniform_cube(1500, 1), 10)
        with pytest.raises(ehgp.InvalidArgument):
            srv.submit(workloads.uniform_cube(100, 1), 11)
        rid = srv.submit(workloads.uniform_cube(100, 1), 10)
        assert srv.wait(rid) == 0
        with pytest.raises(ehgp.EhgpError):
            srv.wait(rid + 1000)
