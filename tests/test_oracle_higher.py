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
