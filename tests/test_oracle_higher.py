"""The triple/quad-support oracle pinned against the reference's own
higher-support stream (build_exact_higher_support_stream run to completion,
tests/golden/make_golden.py --higher; the reference needs ~20 s at n = 12):
minimal (well-centred) supports only, events with exact levels, centres,
interior ids and ranks, extra-shell diagnostics on cospherical ties."""
import glob
import json
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle import pyoracle

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "higher_*.json")))


def load_golden_higher(path):
    d = json.load(open(path))
    F = lambda a, b: Fraction(int(a), int(b))
    ev = [(m, tuple(s), r, e, F(ln, ld), tuple(F(x, c[3]) for x in c[:3]), tuple(ids))
          for m, s, r, e, ln, ld, c, ids in d["events"]]
    dg = [(m, tuple(s), sh, w, mr, orr, ex, F(ln, ld), tuple(F(x, c[3]) for x in c[:3]), tuple(ids))
          for m, s, sh, w, mr, orr, ex, ln, ld, c, ids in d["diagnostics"]]
    return np.array(d["points"]), d["K"], {"events": ev, "diagnostics": dg, "status": d["status"]}


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[7:-5] for p in GOLDEN])
def test_restatement_higher_matches_golden(path):
    pts, K, ref = load_golden_higher(path)
    r = pyoracle.higher(pts, K)
    assert r["events"] == ref["events"]
    assert r["diagnostics"] == ref["diagnostics"]
    assert ref["status"] == "complete"


def test_golden_higher_has_diagnostics():
    assert sum(len(load_golden_higher(p)[2]["diagnostics"]) for p in GOLDEN) > 0


def test_oracle_classify_agrees_with_the_streams():
    """oracle.classify (every point, no pruning) reproduces the interior ids, shell counts
    and least extra-shell witnesses of the restatement's pair and higher streams."""
    rng = np.random.Generator(np.random.PCG64(61))
    p = rng.random((40, 3))
    p[:20] = np.round(p[:20] * 3) / 3  # cospherical ties: extra shells
    pts = np.unique(p, axis=0)
    snap = pyoracle.lbvh_build(pts)
    P = pts[snap["source_index"].astype(np.int64)]
    hi = pyoracle.higher(P, 10)
    pa = pyoracle.pairs(P, 10)
    rows, want = [], []
    for m, ids, rank, ext, lev, cen, inter in hi["events"]:
        rows.append([m, *ids, *([0] * (4 - m))])
        want.append((len(inter), m, 0xffffffff, inter))
    for m, ids, shell, wit, mr, orr, ext, lev, cen, inter in hi["diagnostics"]:
        rows.append([m, *ids, *([0] * (4 - m))])
        want.append((len(inter), shell, wit, inter))
    for u, v, rank, ext, lev, cen, inter in pa["events"]:
        rows.append([2, u, v, 0, 0])
        want.append((len(inter), 2, 0xffffffff, inter))
    for u, v, shell, wit, mr, orr, ext, lev, cen, inter in pa["diagnostics"]:
        rows.append([2, u, v, 0, 0])
        want.append((len(inter), shell, wit, inter))
    assert len(hi["diagnostics"]) + len(pa["diagnostics"]) > 0
    cls = pyoracle.classify(P, np.array(rows, np.uint32))
    for row, w in zip(cls, want):
        I, shell, wit, inter = w
        assert row[0] == 0
        assert (row[1], row[2], row[3]) == (I, shell, wit)
        assert tuple(int(x) for x in row[4:4 + I]) == tuple(inter)


def test_restatement_agrees_with_reference_predicate_tool():
    """The restatement's exact classification (oracle.classify) gives the reference replay
    tool's answers on its support-sphere and support-status fixtures (sizes 2-4, distinct
    points; golden/predicates_ref.json)."""
    import json
    cases = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "predicates_ref.json")))
    assert len(cases) >= 39
    checked = 0
    for case in cases:
        kind = case["predicate"]
        if kind not in ("support_sphere_side", "circumcenter_support_analysis", "binary64_circumcenter_support_analysis"):
            continue
        groups = case["groups"]
        pts_hex = groups["support"] + groups["point"] if kind == "support_sphere_side" else groups["points"]
        pts = np.array([np.array([int(h, 16) for h in p], np.uint64).view(np.float64) + 0.0 for p in pts_hex])
        size = len(groups["support"]) if kind == "support_sphere_side" else len(pts)
        if size < 2 or len(np.unique(pts, axis=0)) != len(pts):
            continue
        snap = pyoracle.lbvh_build(pts)
        P = pts[snap["source_index"].astype(np.int64)]
        pid = np.empty(len(pts), np.int64)
        pid[snap["source_index"].astype(np.int64)] = np.arange(len(pts))
        sup = [int(pid[i]) for i in range(size)]
        row = np.array([[size, *sup, *([0] * (4 - size))]], np.uint32)
        cls = pyoracle.classify(P, row)[0]
        ref = case["reference"]
        if kind == "support_sphere_side":
            if cls[0] != 0:
                continue  # the classification applies to minimal supports only
            side = -1 if cls[1] == 1 else (0 if cls[2] > size else 1)
            assert side == {"negative": -1, "zero": 0, "positive": 1}[ref["sign"]], case["fixture"]
        else:
            assert (cls[0] == 0) == (ref["support_status"] == "minimal"), case["fixture"]
        checked += 1
    assert checked >= 15
