"""The k-NN / EMST / k=1 forest oracle pinned against the reference.

* the restatement (oracle/ehgp_oracle.cpp: brute-force exact top-k with the
  TopKPartition rules, Boruvka rounds with frozen least-PointId labels, the
  compact k=1 forest) against golden fixtures produced by the reference's own
  lbvh_top_k / build_exact_lbvh_boruvka / build_compact_k1_forest
  (tests/golden/make_golden.py --geom);
* the restatement against the reference's code itself (oracle/_ref) on more
  seeded clouds, including exact equality shells and multifusions.
"""
import glob
import os

import numpy as np
import pytest

import workloads
from oracle import pyoracle
from geomcheck import load_golden

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "geom_*.json")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[5:-5] for p in GOLDEN])
def test_restatement_knn_matches_golden(path):
    g = load_golden(path)
    assert pyoracle.knn(g["points"], 11) == g["knn11"]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[5:-5] for p in GOLDEN])
def test_restatement_emst_forest_matches_golden(path):
    g = load_golden(path)
    r = pyoracle.emst_forest(g["points"])
    for k, v in g["emst"].items():
        assert r[k] == v, k


def test_golden_geometry_covers_ties_and_multifusions():
    g = load_golden([p for p in GOLDEN if "grid" in p][0])
    assert any(len(sh) > 1 for _, sh, _ in g["knn11"])          # complete equality shells
    assert max(n[3] for n in g["emst"]["nodes"]) >= 3            # a multifusion


@pytest.mark.skipif(not pyoracle.available("reference"), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", range(3))
def test_restatement_matches_reference_code(seed):
    rng = np.random.Generator(np.random.PCG64(300 + seed))
    pts = rng.random((90, 3))
    pts[:30] = np.round(pts[:30] * 3) / 3
    pts = np.unique(pts, axis=0)
    for k in (1, 4, 11):
        assert pyoracle.knn(pts, k) == pyoracle.knn(pts, k, "reference")
    a, b = pyoracle.emst_forest(pts), pyoracle.emst_forest(pts, "reference")
    for key in b:
        assert a[key] == b[key], key
