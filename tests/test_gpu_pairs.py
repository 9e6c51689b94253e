"""Parity of the sm_100a pair-support enumeration (ehgp_pairs) with the
oracle: the complete set of relevant pair supports, record by record (exact
levels and centres, sorted interior ids, closed ranks, exterior counts,
complete extra shells and their least witness)."""
import glob
import os

import numpy as np
import pytest

import workloads
from oracle import pyoracle
from geomcheck import gpu_pair_records, load_golden_pairs, pairs_match

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "pairs_*.json")))


def canonical(ctx, pts):
    snap = ctx.lbvh_build(pts)
    return np.asarray(pts, dtype=np.float64)[snap.source_index.astype(np.int64)]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[6:-5] for p in GOLDEN])
def test_gpu_pairs_match_golden(ctx, path):
    pts, K, ref = load_golden_pairs(path)
    P = canonical(ctx, pts)
    pairs_match(gpu_pair_records(ctx, K, P), ref)


def _clouds():
    yield "uniform256", workloads.uniform_cube(256, 0)
    yield "uniform1500", workloads.uniform_cube(1500, 7)
    yield "lattice9_f32", workloads.jittered_lattice(9, 2)
    rng = np.random.Generator(np.random.PCG64(43))
    p = rng.random((700, 3))
    p[:350] = np.round(p[:350] * 5) / 5  # cospherical ties: diagnostics
    yield "ties700", np.unique(p, axis=0)
    yield "clustered2000", workloads.clustered(2000, 5)


@pytest.mark.parametrize("name,pts", list(_clouds()), ids=[n for n, _ in _clouds()])
@pytest.mark.parametrize("K", [10, 3])
def test_gpu_pairs_match_oracle(ctx, name, pts, K):
    P = canonical(ctx, pts)
    pairs_match(gpu_pair_records(ctx, K, P), pyoracle.pairs(P, K))
