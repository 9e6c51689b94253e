"""The LBVH oracle pinned against the reference.

* the restatement (oracle/ehgp_oracle.cpp) against the committed golden
  fixtures, which were produced by the reference's own code
  (tests/golden/make_golden.py);
* the restatement against the reference's code itself (oracle/_ref), when it
  has been built, on more seeded clouds;
* the known answers of morsehgp3d/tests/unit/test_spatial_lbvh.cpp:641-744.
"""
import glob
import os

import numpy as np
import pytest

from oracle import pyoracle
import workloads

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "lbvh_*.npz")))
FIELDS = ("source_index", "leaves", "nodes", "counters", "root_aabb")


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[5:-4] for p in GOLDEN])
def test_restatement_matches_golden(path):
    g = np.load(path)
    r = pyoracle.lbvh_build(g["points"], "restatement")
    for k in FIELDS:
        assert np.array_equal(r[k], g[k]), k
    assert r["root"] == int(g["root"])


def test_golden_set_is_present():
    assert len(GOLDEN) >= 7


def test_known_answer_three_way_collision():
    tiny = np.nextafter(0.0, 1.0)
    pts = np.array([[1, 1, 1], [2 * tiny, 0, 0], [0, 0, 0], [tiny, 0, 0]], float)
    r = pyoracle.lbvh_build(pts, "restatement")
    leaves = [tuple(map(int, x)) for x in r["leaves"]]
    assert leaves == [(0, 0), (0, 1), (0, 2), ((2**64 - 1) >> 1, 3)]
    c = r["counters"]
    assert c[0] == 4 and c[1] == 7 and 2 <= c[2] <= 3 and c[3] == 1 and c[4] == 3
    one = np.float64(1.0).view(np.uint64)
    assert list(r["root_aabb"]) == [0, 0, 0, one, one, one]
    # input permutation cannot change the result
    r2 = pyoracle.lbvh_build(pts[[3, 2, 0, 1]], "restatement")
    for k in ("leaves", "nodes", "counters", "root_aabb"):
        assert np.array_equal(r[k], r2[k])


def test_known_answer_finite_extrema():
    tiny, big = np.nextafter(0.0, 1.0), np.finfo(np.float64).max
    pts = np.array([[-big, -tiny, 0], [tiny, big, -big], [big, 0, tiny], [0, -big, big]], float)
    r = pyoracle.lbvh_build(pts, "restatement")
    nb, b = np.float64(-big).view(np.uint64), np.float64(big).view(np.uint64)
    assert list(r["root_aabb"]) == [nb] * 3 + [b] * 3


@pytest.mark.parametrize("bad,msg", [
    (np.array([[0.0, 0, 0], [-0.0, 0, 0]]), "duplicate"),
    (np.array([[np.nan, 0, 0]]), "finite"),
    (np.array([[0.0, np.inf, 0]]), "finite"),
])
def test_restatement_rejects(bad, msg):
    with pytest.raises(pyoracle.OracleError, match=msg):
        pyoracle.lbvh_build(bad, "restatement")


@pytest.mark.skipif(not pyoracle.available("reference"), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", range(4))
def test_restatement_matches_reference_code(seed):
    rng = np.random.Generator(np.random.PCG64(100 + seed))
    n = int(rng.integers(1, 3000))
    pts = rng.random((n, 3)) * 10 ** rng.uniform(-5, 5)
    snap = rng.random(n) < 0.3  # coarse grid: exact ties and Morton collisions
    pts[snap] = np.round(pts[snap] * 64.0) / 64.0 + rng.random((int(snap.sum()), 3)) * 1e-12
    pts = np.unique(pts, axis=0)
    a = pyoracle.lbvh_build(pts, "restatement")
    b = pyoracle.lbvh_build(pts, "reference")
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.skipif(not pyoracle.available("reference"), reason="oracle/_ref not built")
def test_restatement_matches_reference_code_lattice():
    pts = workloads.jittered_lattice(20, 5).astype(np.float64)
    a = pyoracle.lbvh_build(pts, "restatement")
    b = pyoracle.lbvh_build(pts, "reference")
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), k
