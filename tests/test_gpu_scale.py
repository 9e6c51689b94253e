"""Parity of the device chain beyond the small fixtures.

* The plain one-cloud workload itself (256 i.i.d. uniform points, seeds 0-9, K = 10), a 6^3
  jittered lattice and 256-point samples of the clustered generator (with and without the
  2^-10 snapping that forces exact ties) run through the triple/quad supports and the whole
  direct hierarchy; both must equal the restatement oracle exactly.  The oracle's records
  and hierarchy text are pinned as SHA-256 digests in golden/scale_digests.json
  (golden/make_golden.py --scale); the hierarchy comparison is the complete text of facade,
  journal, seeds, forest nodes, children, births, bindings, saddles, groups, batches and
  roots with exact levels.
* Completeness at 1,000 points (golden/scale_higher_digests.json, make_golden.py
  --scale-higher): the device's triple/quad stream on a 1,000-point i.i.d. uniform cloud and a
  10^3 jittered lattice equals the restatement's brute force over every tuple, an enumerator
  that shares neither the direction tables nor the candidate sets of the device.
* The hierarchy's host schedule (chunk size of the parallel record rebuild, descent parts,
  host threads) never changes its result (n = 4096, chunks of 7 batches, parts of 3000 arms).
* Soundness at the regular volumetric workload's size (37^3 = 50,653 jittered lattice points):
  10^4 sampled triple/quad records and 10^4 pair records are classified again exactly against
  every point by the oracle (no bound, no pruning): interior ids, shell counts and witnesses
  must be those the device emitted.
* The clustered, near-degenerate workload at full size (200,000 points, 5 % snapped): the
  chain completes its supports without a capacity failure and the journal refuses with the
  reference's no_journal_relevant_extra_shell_diagnostics decision; sampled diagnostics are
  checked exactly.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import ehgp
import workloads
from geomcheck import gpu_higher_records, gpu_hierarchy_text, hierarchy_diff
from oracle import pyoracle

pytestmark = pytest.mark.gpu

SCALE_PATH = os.path.join(os.path.dirname(__file__), "golden", "scale_digests.json")
# the fixture's presence and completeness are checked on the CPU (test_oracle_hier.py)
SCALE = json.load(open(SCALE_PATH)) if os.path.exists(SCALE_PATH) else {}


SCALE_HIGHER_PATH = os.path.join(os.path.dirname(__file__), "golden", "scale_higher_digests.json")
SCALE_HIGHER = json.load(open(SCALE_HIGHER_PATH)) if os.path.exists(SCALE_HIGHER_PATH) else {}


def higher_digest(rec):
    return hashlib.sha256(repr((rec["events"], rec["diagnostics"])).encode()).hexdigest()


def canonical(ctx, pts):
    snap = ctx.lbvh_build(pts)
    return np.asarray(pts, dtype=np.float64)[snap.source_index.astype(np.int64)]


@pytest.mark.parametrize("name", list(SCALE))
def test_gpu_higher_matches_restatement_at_scale(ctx, name):
    d = SCALE[name]
    P = canonical(ctx, np.array(d["points"]))
    rec = gpu_higher_records(ctx, d["K"], P)
    assert (len(rec["events"]), len(rec["diagnostics"])) == (d["higher_events"], d["higher_diagnostics"])
    assert higher_digest(rec) == d["higher_sha256"]


@pytest.mark.parametrize("name", list(SCALE_HIGHER))
def test_gpu_higher_complete_at_1000_points(ctx, name):
    d = SCALE_HIGHER[name]
    P = canonical(ctx, np.array(d["points"]))
    rec = gpu_higher_records(ctx, d["K"], P)
    assert (len(rec["events"]), len(rec["diagnostics"])) == (d["higher_events"], d["higher_diagnostics"])
    assert higher_digest(rec) == d["higher_sha256"]


@pytest.mark.parametrize("name", list(SCALE))
def test_gpu_hierarchy_matches_restatement_at_scale(ctx, name):
    d = SCALE[name]
    ctx.lbvh_build(np.array(d["points"]), outputs=False)
    if d["refused"]:
        with pytest.raises(ehgp.DegenerateError):
            ctx.hierarchy(d["K"])
        c = ctx.last_hier_counts
        assert (c["events"], c["diagnostics"]) == (d["facade_events"], d["diagnostics"])
        return
    text = gpu_hierarchy_text(ctx, d["K"])
    lines = text.splitlines()
    assert (len(lines), lines[-1]) == (d["hierarchy_lines"], d["hierarchy_last"])
    assert hashlib.sha256(text.encode()).hexdigest() == d["hierarchy_sha256"]


HIER_ARRAYS = ("events", "journal_batches", "roles", "families", "arm_removed", "nodes", "children", "births",
               "bindings", "saddles", "groups", "batches", "roots", "vertical")


def test_gpu_hierarchy_schedule_does_not_change_result(ctx):
    """Many small chunks and descent parts on three host threads, and one chunk and one
    part per order on one thread, give the default schedule's records exactly."""
    pts = workloads.jittered_lattice(16, 1).astype(np.float64)
    ctx.lbvh_build(pts, outputs=False)
    base = ctx.hierarchy(10)
    try:
        ctx.hier_schedule(chunk_batches=7, part_arms=3000, host_threads=3)
        forced = ctx.hierarchy(10)
        ctx.hier_schedule(chunk_batches=1 << 30, part_arms=1 << 30, host_threads=1)
        single = ctx.hierarchy(10)
    finally:
        ctx.hier_schedule(0, 0, 0)
    for key in HIER_ARRAYS:
        assert np.array_equal(base[key], forced[key]), key
        assert np.array_equal(base[key], single[key]), key


def test_gpu_hierarchy_forced_schedule_matches_restatement(ctx):
    pts = np.random.default_rng(12).random((48, 3))
    ctx.lbvh_build(pts, outputs=False)
    try:
        ctx.hier_schedule(chunk_batches=1, part_arms=5, host_threads=2)
        got = gpu_hierarchy_text(ctx, 10)
    finally:
        ctx.hier_schedule(0, 0, 0)
    want = pyoracle.hierarchy(pts, 10)
    assert got == want, hierarchy_diff(got, want)


def _check_classified(sup, cls, interior_count, shell_count, witness, interior_ids, width):
    assert np.all(cls[:, 0] == 0), "a sampled record is not a minimal support"
    assert np.array_equal(cls[:, 1], interior_count)
    assert np.array_equal(cls[:, 2], shell_count)
    extra = shell_count > sup[:, 0]
    assert np.array_equal(cls[extra, 3], witness[extra])
    for i in range(len(sup)):
        I = int(interior_count[i])
        assert np.array_equal(cls[i, 4:4 + min(I, width)], interior_ids[i, :min(I, width)])


def test_gpu_supports_sound_at_50k_lattice(ctx):
    pts = workloads.jittered_lattice(37, 0)
    P = canonical(ctx, pts)
    rng = np.random.default_rng(5)
    hr = ctx.higher(10)
    pick = np.sort(rng.choice(len(hr), size=min(10_000, len(hr)), replace=False))
    h = hr[pick]
    sup = np.c_[h["size"], h["ids"]].astype(np.uint32)
    cls = pyoracle.classify(P, sup)
    _check_classified(sup, cls, h["interior_count"], h["shell_count"], h["extra_shell_witness"], h["interior_ids"], 8)
    pr = ctx.pairs(10)["records"]
    pick = np.sort(rng.choice(len(pr), size=min(10_000, len(pr)), replace=False))
    p = pr[pick]
    sup = np.c_[np.full(len(p), 2), p["u"], p["v"], np.zeros((len(p), 2))].astype(np.uint32)
    cls = pyoracle.classify(P, sup)
    _check_classified(sup, cls, p["interior_count"], p["shell_count"], p["extra_shell_witness"], p["interior_ids"], 9)


@pytest.mark.skipif(os.environ.get("EHGP_GPU_FULL_CLUSTERED") != "1",
                    reason="about 7 minutes on one B200: set EHGP_GPU_FULL_CLUSTERED=1")
def test_gpu_clustered_200k_refused_by_the_journal(ctx):
    """The clustered near-degenerate workload at its full size (200,000 points): its supports
    complete (large neighbourhoods and large candidate sets included) and the journal refuses."""
    pts = workloads.clustered(200_000, 0)
    P = canonical(ctx, pts)
    with pytest.raises(ehgp.DegenerateError):
        ctx.hierarchy(10)
    c = ctx.last_hier_counts
    assert c["diagnostics"] > 0 and c["events"] > 0
    _check_clustered_diagnostics(ctx, P, c)


def test_gpu_clustered_20k_completes(ctx):
    """20,000 points of the clustered generator (5 % snapped): owners on cluster edges take
    the large-neighbourhood path and large candidate sets; the supports complete, sampled
    records are exact against every point, and the hierarchy completes or is refused by the
    journal (never a capacity failure)."""
    pts = workloads.clustered(20_000, 0)
    P = canonical(ctx, pts)
    hr = ctx.higher(10)
    _, st = ctx.higher_stats()
    assert int(st[8]) > 0 and int(st[10]) > 0
    rng = np.random.default_rng(21)
    h = hr[np.sort(rng.choice(len(hr), size=min(3000, len(hr)), replace=False))]
    sup = np.c_[h["size"], h["ids"]].astype(np.uint32)
    _check_classified(sup, pyoracle.classify(P, sup), h["interior_count"], h["shell_count"],
                      h["extra_shell_witness"], h["interior_ids"], 8)
    try:
        r = ctx.hierarchy(10, arrays=False)
        assert r["decision"] == 0 and r["final_roots"] == 10
    except ehgp.DegenerateError:
        _check_clustered_diagnostics(ctx, P, ctx.last_hier_counts)


def _check_clustered_diagnostics(ctx, P, c):
    # sampled extra-shell diagnostics, classified again exactly against every point
    rng = np.random.default_rng(9)
    hr = ctx.higher(10)
    diag = hr[hr["shell_count"] > hr["size"]]
    pr = ctx.pairs(10)["records"]
    pdiag = pr[pr["shell_count"] > 2]
    assert len(diag) + len(pdiag) == c["diagnostics"]
    if len(diag):
        h = diag[np.sort(rng.choice(len(diag), size=min(200, len(diag)), replace=False))]
        sup = np.c_[h["size"], h["ids"]].astype(np.uint32)
        _check_classified(sup, pyoracle.classify(P, sup), h["interior_count"], h["shell_count"],
                          h["extra_shell_witness"], h["interior_ids"], 8)
    if len(pdiag):
        p = pdiag[np.sort(rng.choice(len(pdiag), size=min(200, len(pdiag)), replace=False))]
        sup = np.c_[np.full(len(p), 2), p["u"], p["v"], np.zeros((len(p), 2))].astype(np.uint32)
        _check_classified(sup, pyoracle.classify(P, sup), p["interior_count"], p["shell_count"],
                          p["extra_shell_witness"], p["interior_ids"], 9)


def test_gpu_record_buffers_grow_on_demand(ctx):
    """count -> allocate -> emit: with the pair and triple/quad record buffers shrunk to 16
    records, both stages grow them and run again, and the records equal those of the
    ample buffers."""
    pts = workloads.jittered_lattice(12, 4)
    canonical(ctx, pts)
    want_p = ctx.pairs(10)["records"].copy()
    want_h = ctx.higher(10).copy()
    before = ctx.regrowths()
    ctx.reserve(0, 16)
    ctx.reserve(1, 16)
    ctx.lbvh_build(pts, outputs=False)
    got_p = ctx.pairs(10)["records"]
    got_h = ctx.higher(10)
    assert ctx.regrowths() >= before + 2
    assert np.array_equal(got_p, want_p)
    assert np.array_equal(got_h, want_h)


def _higher_clouds():
    yield "uniform64", workloads.uniform_cube(64, 1)
    yield "lattice4_f32", workloads.jittered_lattice(4, 3)
    rng = np.random.Generator(np.random.PCG64(44))
    p = rng.random((60, 3))
    p[:30] = np.round(p[:30] * 3) / 3  # cospherical ties
    yield "ties60", np.unique(p, axis=0)
    yield "clustered70", workloads.clustered(70, 6)


@pytest.mark.parametrize("name,pts", list(_higher_clouds()), ids=[n for n, _ in _higher_clouds()])
def test_gpu_large_neighbourhood_path_matches_restatement(ctx, name, pts):
    """With the list capacity lowered to 8 entries, nearly every owner certifies its direction
    table on the large-neighbourhood path (arena lists, unsorted chunked scan); the records
    equal the restatement's."""
    from geomcheck import higher_match
    P = canonical(ctx, pts)
    try:
        ctx.tune(ctx.TUNE_HIGHER_LIST, 8)
        got = gpu_higher_records(ctx, 10, P)
        _, st = ctx.higher_stats()
    finally:
        ctx.tune(ctx.TUNE_HIGHER_LIST, 1024)
    assert int(st[8]) > len(P) // 2
    higher_match(got, pyoracle.higher(P, 10))


def test_gpu_dense_cluster_in_sparse_background(ctx):
    """A dense cluster inside a sparse background: owners on the cluster's edge need more
    neighbours than a list holds (their bounds reach into the background); the stage
    completes, and its records equal those of the run where every owner takes the large path."""
    rng = np.random.Generator(np.random.PCG64(71))
    pts = np.unique(np.r_[rng.normal(5.0, 0.06, (1500, 3)), rng.uniform(0, 10, (250, 3))], axis=0)
    canonical(ctx, pts)
    h = ctx.higher(10).copy()
    _, st = ctx.higher_stats()
    assert int(st[8]) > 0
    try:
        ctx.tune(ctx.TUNE_HIGHER_LIST, 64)
        ctx.lbvh_build(pts, outputs=False)
        h1 = ctx.higher(10)
    finally:
        ctx.tune(ctx.TUNE_HIGHER_LIST, 1024)
    assert np.array_equal(h, h1)
