"""The pair-support oracle pinned against the reference's own pair stream.

The restatement (oracle/ehgp_oracle.cpp: every pair, exact diametral-sphere
sides) must reproduce build_exact_pair_support_stream run to completion
(golden fixtures from tests/golden/make_golden.py --pairs, which runs the
reference's code): events with exact levels, centres, interior ids and ranks,
and extra-shell diagnostics with complete shell counts and least witnesses."""
import glob
import os

import pytest

from oracle import pyoracle
from geomcheck import load_golden_pairs, pairs_match

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "pairs_*.json")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[6:-5] for p in GOLDEN])
def test_restatement_pairs_match_golden(path):
    pts, K, ref = load_golden_pairs(path)
    pairs_match(pyoracle.pairs(pts, K), ref)


def test_golden_pairs_cover_events_and_diagnostics():
    totals = [load_golden_pairs(p)[2] for p in GOLDEN]
    assert sum(len(t["events"]) for t in totals) > 2000
    assert sum(len(t["diagnostics"]) for t in totals) > 500


@pytest.mark.parametrize("K", [1, 2, 4])
def test_restatement_small_orders(K):
    import workloads
    pts = workloads.uniform_cube(40, 9)
    r = pyoracle.pairs(pts, K)
    smax = min(min(K, 40) + 1, 40)
    assert all(e[2] <= smax for e in r["events"])
