"""The reference's predicate fixtures (morsehgp3d/tests/fixtures/predicates/: one-ulp boundaries,
cancellations, subnormal and extreme exponents) against the device's exact predicates.

The answers come from the reference's own replay tool (morsehgp3d/src/tools/predicate_replay.cpp,
compiled unmodified into oracle/_ref; golden/predicates_ref.json, make_golden.py --predicates).
Each fixture's points become a cloud; ehgp_predicate_eval runs the enumeration's helpers on
their PointIds (FP64 with the uniform error bounds, fixed-width exact integers where the filter
does not decide).  A cloud outside the device's exact fixed-point range (|x 2^S| < 2^124) must
be refused with EHGP_ERR_NUMERIC_RANGE, never answered wrongly.
"""
import json
import os

import numpy as np
import pytest

import ehgp

pytestmark = pytest.mark.gpu

CASES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "predicates_ref.json")))
STATUS = {"minimal": 0, "boundary_reduced": 1, "exterior_circumcenter": 2, "affinely_dependent": 3}
SIGN = {"negative": -1, "zero": 0, "positive": 1}


def point(hexes):
    v = np.array([int(h, 16) for h in hexes], dtype=np.uint64).view(np.float64)
    return v + 0.0  # -0 -> +0, as the canonical cloud does


def cloud_of(groups):
    """Distinct points of the fixture as a cloud, and each group's indices into it."""
    keys, pts, idx = {}, [], {}
    for g, plist in groups.items():
        idx[g] = []
        for h in plist:
            p = point(h)
            k = p.tobytes()
            if k not in keys:
                keys[k] = len(pts)
                pts.append(p)
            idx[g].append(keys[k])
    return np.array(pts), idx


@pytest.fixture(scope="module")
def pctx():
    c = ehgp.Context(max_points=16)
    yield c
    c.close()


@pytest.mark.parametrize("case", CASES, ids=[c["fixture"][:-5] for c in CASES])
def test_gpu_predicate_matches_reference_tool(pctx, case):
    ref = case["reference"]
    assert "error" not in ref
    cloud, idx = cloud_of(case["groups"])
    snap = pctx.lbvh_build(cloud)
    pid = np.empty(len(cloud), np.int64)
    pid[snap.source_index.astype(np.int64)] = np.arange(len(cloud))
    P = {g: [int(pid[i]) for i in v] for g, v in idx.items()}
    kind = case["predicate"]
    if kind == "support_sphere_side":
        args, code = P["support"] + P["point"], pctx.PRED_SUPPORT_SIDE
    elif kind == "compare_support_levels":
        args, code = [len(P["left"])] + P["left"] + P["right"], pctx.PRED_LEVEL_CMP
    elif kind == "compare_squared_distances":
        args, code = P["points"], pctx.PRED_DISTANCE_CMP
    else:
        args, code = P["points"], pctx.PRED_SUPPORT_STATUS
    _, valid = pctx.scale()
    if not valid:
        with pytest.raises(ehgp.NumericRange):
            pctx.predicate(code, args)
        pytest.skip("outside the device's exact fixed-point range (refused, as documented)")
    got, _ = pctx.predicate(code, args)
    if code == pctx.PRED_SUPPORT_STATUS:
        assert got == STATUS[ref["support_status"]]
    else:
        assert got == SIGN[ref["sign"]]


def test_gpu_predicate_fixtures_mostly_in_range(pctx):
    """The fixed-point range excludes few of the reference's fixtures."""
    inside = 0
    for case in CASES:
        cloud, _ = cloud_of(case["groups"])
        pctx.lbvh_build(cloud, outputs=False)
        inside += pctx.scale()[1]
    assert inside >= len(CASES) - 8, inside
