"""Parity of the sm_100a triple/quad-support enumeration (ehgp_higher) with
the oracle: every relevant minimal support, record by record (exact levels
and centres recomputed from the ids, sorted interior ids, ranks, complete
extra shells and their least witness)."""
import glob
import os

import numpy as np
import pytest

import workloads
from oracle import pyoracle
from geomcheck import gpu_higher_records, higher_match
from test_oracle_higher import load_golden_higher

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "higher_*.json")))


def canonical(ctx, pts):
    snap = ctx.lbvh_build(pts)
    return np.asarray(pts, dtype=np.float64)[snap.source_index.astype(np.int64)]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[7:-5] for p in GOLDEN])
def test_gpu_higher_matches_golden(ctx, path):
    pts, K, ref = load_golden_higher(path)
    P = canonical(ctx, pts)
    higher_match(gpu_higher_records(ctx, K, P), ref)


def _clouds():
    yield "uniform64", workloads.uniform_cube(64, 1)
    yield "lattice4_f32", workloads.jittered_lattice(4, 3)
    rng = np.random.Generator(np.random.PCG64(44))
    p = rng.random((60, 3))
    p[:30] = np.round(p[:30] * 3) / 3  # cospherical ties
    yield "ties60", np.unique(p, axis=0)
    yield "clustered70", workloads.clustered(70, 6)


@pytest.mark.parametrize("name,pts", list(_clouds()), ids=[n for n, _ in _clouds()])
@pytest.mark.parametrize("K", [10, 5])
def test_gpu_higher_matches_oracle(ctx, name, pts, K):
    P = canonical(ctx, pts)
    higher_match(gpu_higher_records(ctx, K, P), pyoracle.higher(P, K))
