"""Parity of the sm_100a LBVH build (C ABI ehgp_lbvh_build) with the oracle.

Bit-exact on every field of the reference's MortonLbvhSnapshot: canonical
source permutation, (code, PointId) leaves, postorder nodes with ranges,
children and the six AABB witness PointIds, counters and the root AABB.
Where oracle/_ref is present, the reference's own exhaustive validator
(MortonLbvhIndex::import_certified_snapshot) must also accept the GPU
snapshot.
"""
import glob
import os

import numpy as np
import pytest

import ehgp
import workloads
from oracle import pyoracle

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "lbvh_*.npz")))
FIELDS = ("source_index", "leaves", "nodes", "counters", "root_aabb")


def assert_same(snap, ref):
    for k in FIELDS:
        got = getattr(snap, k)
        assert got.shape == ref[k].shape, k
        if not np.array_equal(got, ref[k]):
            bad = np.nonzero((got != ref[k]).reshape(len(got), -1).any(1))[0]
            raise AssertionError(f"{k} differs at {bad[:10]} (of {len(bad)})")
    assert snap.root == ref["root"]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[5:-4] for p in GOLDEN])
def test_gpu_matches_golden(ctx, path):
    g = np.load(path)
    snap = ctx.lbvh_build(g["points"])
    assert_same(snap, {k: g[k] for k in FIELDS} | {"root": int(g["root"])})


@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (3, 2), (17, 3), (1000, 4), (4097, 5), (65_537, 6)])
def test_gpu_matches_oracle_uniform(ctx, n, seed):
    pts = workloads.uniform_cube(n, seed)
    snap = ctx.lbvh_build(pts)
    assert_same(snap, pyoracle.lbvh_build(pts))


def test_gpu_matches_oracle_lattice_f32(ctx):
    pts = workloads.jittered_lattice(37, 0)
    snap = ctx.lbvh_build(pts)  # binary32 entry point, widened exactly on the device
    assert_same(snap, pyoracle.lbvh_build(pts.astype(np.float64)))


def test_gpu_matches_oracle_clustered(ctx):
    pts = workloads.clustered(200_000, 0)
    snap = ctx.lbvh_build(pts)
    assert_same(snap, pyoracle.lbvh_build(pts))


def test_gpu_collision_groups(ctx):
    rng = np.random.Generator(np.random.PCG64(11))
    pts = rng.random((5000, 3))
    pts[:2500] = np.round(pts[:2500] * 3) / 3 + rng.random((2500, 3)) * 1e-10
    snap = ctx.lbvh_build(pts)
    ref = pyoracle.lbvh_build(pts)
    assert ref["counters"][3] > 0
    assert_same(snap, ref)


def test_gpu_input_permutation_invariant(ctx):
    pts = workloads.uniform_cube(3000, 9)
    a = ctx.lbvh_build(pts)
    perm = np.random.Generator(np.random.PCG64(1)).permutation(len(pts))
    b = ctx.lbvh_build(pts[perm])
    for k in ("leaves", "nodes", "counters", "root_aabb"):
        assert np.array_equal(getattr(a, k), getattr(b, k))
    assert np.array_equal(perm[b.source_index.astype(np.int64)], a.source_index.astype(np.int64))


@pytest.mark.skipif(not pyoracle.available("reference"), reason="oracle/_ref not built")
@pytest.mark.parametrize("maker", ["uniform", "spread"])
def test_reference_certifies_gpu_snapshot(ctx, maker):
    if maker == "uniform":
        pts = workloads.uniform_cube(20_000, 3)
    else:
        rng = np.random.Generator(np.random.PCG64(5))
        pts = rng.random((2000, 3)) * 1e-200
        pts[:10] *= 1e300  # far points: exponent spread ~1600 bits
    snap = ctx.lbvh_build(pts)
    ok, msg = pyoracle.ref_lbvh_certify(pts, snap)
    assert ok, msg


@pytest.mark.parametrize("bad,exc", [
    (np.array([[0.0, 0, 0], [-0.0, 0, 0]]), ehgp.DuplicatePoint),
    (np.array([[1.0, 2.0, 3.0], [1.0, 2.0, 3.0], [0, 0, 0]]), ehgp.DuplicatePoint),
    (np.array([[np.nan, 0, 0], [1, 1, 1]]), ehgp.InvalidArgument),
    (np.array([[0.0, np.inf, 0]]), ehgp.InvalidArgument),
    (np.zeros((0, 3)), ehgp.InvalidArgument),
])
def test_gpu_rejects_like_reference(ctx, bad, exc):
    with pytest.raises(exc):
        ctx.lbvh_build(bad)
    # the context stays usable after a rejected cloud
    pts = workloads.uniform_cube(64, 1)
    assert_same(ctx.lbvh_build(pts), pyoracle.lbvh_build(pts))


def test_gpu_capacity_error():
    with ehgp.Context(max_points=100) as small:
        with pytest.raises(ehgp.CapacityError):
            small.lbvh_build(workloads.uniform_cube(101, 0))
