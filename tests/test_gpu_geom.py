"""Parity of the sm_100a k-NN (ehgp_knn), Boruvka EMST (ehgp_emst) and
compact k=1 forest (ehgp_k1_forest) with the oracle: exact, record by record
(cutoffs and squared lengths as exact rationals, complete equality shells,
per-round component minima, multifusion nodes, batches)."""
import glob
import os
from fractions import Fraction

import numpy as np
import pytest

import ehgp
import workloads
from oracle import pyoracle
from geomcheck import (emst_forest_matches, gpu_emst_forest, gpu_knn_records, knn_matches, load_golden)

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "geom_*.json")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[5:-5] for p in GOLDEN])
def test_gpu_geometry_matches_golden(ctx, path):
    g = load_golden(path)
    ctx.lbvh_build(g["points"], outputs=False)
    knn_matches(gpu_knn_records(ctx, 11), g["knn11"], 11)
    emst_forest_matches(gpu_emst_forest(ctx), g["emst"])


def _clouds():
    yield "uniform256", workloads.uniform_cube(256, 0)
    yield "lattice8_f32", workloads.jittered_lattice(8, 2)
    rng = np.random.Generator(np.random.PCG64(41))
    p = rng.random((500, 3))
    p[:250] = np.round(p[:250] * 6) / 6  # exact ties: shells and multifusions
    yield "ties500", np.unique(p, axis=0)
    c = workloads.clustered(600, 3)
    yield "clustered600", c


@pytest.mark.parametrize("name,pts", list(_clouds()), ids=[n for n, _ in _clouds()])
@pytest.mark.parametrize("k", [1, 4, 11])
def test_gpu_knn_matches_oracle(ctx, name, pts, k):
    ctx.lbvh_build(pts, outputs=False)
    knn_matches(gpu_knn_records(ctx, k), pyoracle.knn(pts.astype(np.float64), k), k)


@pytest.mark.parametrize("name,pts", list(_clouds()), ids=[n for n, _ in _clouds()])
def test_gpu_emst_forest_matches_oracle(ctx, name, pts):
    ctx.lbvh_build(pts, outputs=False)
    emst_forest_matches(gpu_emst_forest(ctx), pyoracle.emst_forest(pts.astype(np.float64)))


def _exact_d2(P, S, a, b):
    """Exact squared distance numerator at scale 2^-2S from binary64 coordinates."""
    tot = 0
    for x, y in zip(P[a], P[b]):
        fx, fy = Fraction(float(x)), Fraction(float(y))
        tot += (fx - fy) ** 2
    return tot


def test_gpu_emst_full_size_properties(ctx):
    """50,653-point lattice: spanning tree, exact nondecreasing order, a merge
    forest with one root covering every point."""
    pts = workloads.jittered_lattice(37, 0)
    snap = ctx.lbvh_build(pts)
    P = pts.astype(np.float64)[snap.source_index.astype(np.int64)]  # canonical order
    S, valid = ctx.scale()
    assert valid
    e = ctx.emst(with_minima=False)
    n = len(pts)
    assert len(e["u"]) == n - 1
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x
    for u, v in zip(e["u"], e["v"]):
        assert u < v
        a, b = find(int(u)), find(int(v))
        assert a != b
        parent[max(a, b)] = min(a, b)
    D = [ehgp.limbs_to_int(x) for x in e["D"]]
    keys = list(zip(D, e["u"].tolist(), e["v"].tolist()))
    assert all(keys[i] < keys[i + 1] for i in range(len(keys) - 1))
    rng = np.random.Generator(np.random.PCG64(0))
    for i in rng.choice(n - 1, 200, replace=False):
        assert Fraction(D[i], 1 << (2 * S)) == _exact_d2(P, S, int(e["u"][i]), int(e["v"][i]))
    f = ctx.k1_forest()
    assert f["nodes"].shape[0] >= 1
    root = f["root"]
    assert root >= n and int(f["nodes"][root - n][5]) == n


def test_gpu_knn_full_size_sample(ctx):
    """50,653-point lattice: the exact cutoff of sampled queries equals a
    brute-force exact evaluation against every point."""
    pts = workloads.jittered_lattice(37, 0)
    snap = ctx.lbvh_build(pts)
    P = pts.astype(np.float64)[snap.source_index.astype(np.int64)]
    r = ctx.knn(11)
    S, _ = ctx.scale()
    rng = np.random.Generator(np.random.PCG64(1))
    for p in rng.choice(len(P), 40, replace=False):
        d = ((P - P[p]) ** 2).sum(1)
        d[p] = np.inf
        cand = np.nonzero(d <= np.sort(d)[10] * (1 + 1e-9))[0]
        exact = sorted((_exact_d2(P, S, p, int(q)), int(q)) for q in cand)
        cut = exact[10][0]
        assert r["cutoff"][p] == cut
        strict = [q for x, q in exact if x < cut]
        shell = [q for x, q in exact if x == cut]
        assert list(r["ids"][p][: len(strict)]) == strict
        assert int(r["meta"][p][0]) == len(strict) and int(r["meta"][p][1]) == len(shell)


def test_stages_need_a_resident_cloud():
    with ehgp.Context(max_points=64) as c:
        with pytest.raises(ehgp.EhgpError):
            c.n = 10
            c.knn(3)
