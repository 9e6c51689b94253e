"""The direct-hierarchy oracle (facade -> Morse event journal -> arm seeds ->
forest journal, with strict-arm descent and frozen-root quotient) pinned
against the reference's own chain run to completion
(tests/golden/make_golden.py --hierarchy; the reference needs seconds per
10 points).  Text lines follow oracle/ref_driver.cpp ref_hierarchy."""
import glob
import json
import os

import numpy as np
import pytest

from oracle import pyoracle

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "hier_*.json")))


def load_golden_hier(path):
    d = json.load(open(path))
    return np.array(d["points"]), d["K"], d["text"]


def first_diff(a, b):
    for x, y in zip(a.splitlines(), b.splitlines()):
        if x != y:
            return f"\n  oracle: {x[:200]}\n  golden: {y[:200]}"
    return f"line counts {len(a.splitlines())} vs {len(b.splitlines())}"


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[5:-5] for p in GOLDEN])
def test_restatement_hierarchy_matches_golden(path):
    pts, K, ref = load_golden_hier(path)
    got = pyoracle.hierarchy(pts, K)
    assert got == ref, first_diff(got, ref)


def test_golden_hierarchy_covers_forest_and_refusal():
    texts = [load_golden_hier(p)[2] for p in GOLDEN]
    assert any(t.rstrip().endswith("D 5 5 13") for t in texts)       # complete forests
    assert any(t.rstrip().endswith("D 4 3 4") for t in texts)        # journal refusal on extra shells
    assert any("\nG " in t and " 2\n" in t for t in texts)           # multifusion groups


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(pyoracle.__file__), "_ref", "libehgp_ref.so")),
                    reason="reference build absent")
def test_restatement_hierarchy_matches_live_reference():
    pts = np.random.default_rng(23).random((6, 3))
    a = pyoracle.hierarchy(pts, 10)
    b = pyoracle.hierarchy(pts, 10, which="reference")
    assert a == b, first_diff(a, b)


DEFINITION = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "definition_*.json")))


@pytest.mark.parametrize("path", DEFINITION, ids=[os.path.basename(p)[11:-5] for p in DEFINITION])
def test_restatement_forest_matches_hgp_reduced_definition(path):
    """The direct forest journal's nodes equal the normative hgp_reduced forests of the
    exhaustive-Gamma Python oracle (reference/morsehgp3d_oracle, run_oracle(...,
    profile='hgp_reduced'); tests/golden/make_golden.py --definition): kinds, exact
    levels, children and final roots, order by order."""
    from geomcheck import definition_match, forests_from_hier_text
    d = json.load(open(path))
    text = pyoracle.hierarchy(np.array(d["points"]), d["K"])
    got = forests_from_hier_text(text)
    msg = definition_match(got, d["forests"])
    assert msg == "", msg


@pytest.mark.parametrize("path", DEFINITION, ids=[os.path.basename(p)[11:-5] for p in DEFINITION])
def test_vertical_maps_from_journal_match_definition(path):
    """Vertical maps derived from the direct journal (a group's carrier birth is a saddle
    one order down; its group's root, climbed on the closed cut) equal the contract
    serializer's assignments of the exhaustive-Gamma oracle."""
    from geomcheck import vertical_from_hier_text
    d = json.load(open(path))
    got = vertical_from_hier_text(pyoracle.hierarchy(np.array(d["points"]), d["K"]))
    assert sorted(got) == sorted(d["vertical"])


def test_scale_digest_fixture_is_complete():
    """golden/scale_digests.json (make_golden.py --scale) holds every case of the
    plain-workload parity set: cfg1 seeds 0-9, the 6^3 lattice, clustered samples."""
    import json
    import os
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "scale_digests.json")))
    names = set(d)
    assert {f"uniform256_s{s}" for s in range(10)} <= names
    assert "lattice6_f32" in names
    assert any(k.startswith("clustered256_snap") for k in names)
    assert any(k.startswith("clustered256_s") and "snap" not in k for k in names)
    for k, v in d.items():
        assert len(v["points"]) >= 216 and len(v["higher_sha256"]) == 64 and len(v["hierarchy_sha256"]) == 64, k


def test_scale_higher_fixture_is_complete():
    """golden/scale_higher_digests.json (make_golden.py --scale-higher) holds the restatement's
    complete triple/quad streams of a 1,000-point uniform cloud and a 10^3 jittered lattice."""
    import json
    import os
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "scale_higher_digests.json")))
    assert {"uniform1000_s0", "lattice10_f32"} <= set(d)
    for k, v in d.items():
        assert len(v["points"]) == 1000 and v["K"] == 10 and len(v["higher_sha256"]) == 64, k
        assert v["higher_events"] > 100000, k
