"""Contract-v2 output of the direct hierarchy (MorseHGP3DResult).

Schema: morsehgp3d/schemas/morsehgp3d-contract-v2.schema.json ($defs.MorseHGP3DResult).
Reference writer: reference/morsehgp3d_oracle/serialization.py:199 (serialize_oracle_result),
whose identity rules this module follows where a record's content is the same:
canonical JSON (sorted keys, no whitespace), SHA-256 over "MorseHGP3D/v2/<record type>/"
followed by the record's identity projection without schema_version keys
(serialization.py:24-62), exact levels and rational points as decimal strings
(serialization.py:65-97).

What is exact and what is conditional:
  * critical_catalog: every singleton and every facade event, with the same event ids
    and fields as the reference serializer (checked by the tests);
  * forests, equal_level_batches, vertical_maps: the direct Morse forest journal
    (conditional H0 candidate in the reference's own words), published under
    proof_basis m1_conditional_contract, result_kind partial_hierarchy and
    forest_semantics partial_refinement.  Node coverage lists the points of the
    facets the journal certifies in the component (its birth and saddle events and
    children): a positive guarantee, not the Gamma coverage of the exhaustive oracle.
    Gamma cofaces, Gabriel hyperedges and attachments are not enumerated.

This is a host formatting pass over the hierarchy arrays (exact rationals in Python);
it is not part of the timed device path.
"""
from __future__ import annotations

import hashlib
import json
import struct
from fractions import Fraction
from math import comb, gcd
from typing import Any, Mapping, Sequence

import numpy as np

SCHEMA_VERSION = "2.0.0"
CONTRACT_DOMAIN = "MorseHGP3D/v2"
COORDINATE_UNIT = "input_coordinate_unit"
SQUARED_LEVEL_UNIT = "input_coordinate_unit_squared"
ABSENT = 0xFFFFFFFF


# ---- identity rules -------------------------------------------------------------------
def canonical_json(value: Any) -> str:
    return json.dumps(value, ensure_ascii=False, allow_nan=False, sort_keys=True, separators=(",", ":"))


def _strip_versions(value: Any) -> Any:
    if isinstance(value, Mapping):
        return {k: _strip_versions(v) for k, v in value.items() if k != "schema_version"}
    if isinstance(value, (list, tuple)):
        return [_strip_versions(v) for v in value]
    return value


def canonical_id(record_type: str, projection: Any) -> str:
    h = hashlib.sha256()
    h.update(f"{CONTRACT_DOMAIN}/{record_type}/".encode("ascii"))
    h.update(canonical_json(_strip_versions(projection)).encode("utf-8"))
    return h.hexdigest()


def exact_level(value: Fraction) -> dict:
    v = Fraction(value)
    return {"schema_version": SCHEMA_VERSION, "numerator": str(v.numerator), "denominator": str(v.denominator),
            "unit": SQUARED_LEVEL_UNIT}


def exact_rational3(values: Sequence[Fraction]) -> dict:
    den = 1
    for v in values:
        den = den * v.denominator // gcd(den, v.denominator)
    nums = [v.numerator * (den // v.denominator) for v in values]
    common = den
    for x in nums:
        common = gcd(common, abs(x))
    den //= common
    nums = [x // common for x in nums]
    return {"schema_version": SCHEMA_VERSION, "x_numerator": str(nums[0]), "y_numerator": str(nums[1]),
            "z_numerator": str(nums[2]), "denominator": str(den), "unit": COORDINATE_UNIT}


def binary64_bits(value: float) -> str:
    v = 0.0 if value == 0.0 else float(value)
    return struct.pack(">d", v).hex()


# ---- exact circumspheres ----------------------------------------------------------------
def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def exact_sphere(P: Sequence[tuple], ids: Sequence[int]) -> tuple[tuple, Fraction]:
    """Centre and squared radius of the circumsphere of a 1- to 4-point minimal support."""
    a = P[ids[0]]
    if len(ids) == 1:
        return a, Fraction(0)
    if len(ids) == 2:
        c = tuple((a[i] + P[ids[1]][i]) / 2 for i in range(3))
        return c, _dot(_sub(c, a), _sub(c, a))
    if len(ids) == 3:
        e1, e2 = _sub(P[ids[1]], a), _sub(P[ids[2]], a)
        g11, g12, g22 = _dot(e1, e1), _dot(e1, e2), _dot(e2, e2)
        det = g11 * g22 - g12 * g12
        f1, f2 = g22 * (g11 - g12), g11 * (g22 - g12)
        off = tuple((f1 * e1[i] + f2 * e2[i]) / (2 * det) for i in range(3))
    else:
        e1, e2, e3 = (_sub(P[i], a) for i in ids[1:])
        c23, c31, c12 = _cross(e2, e3), _cross(e3, e1), _cross(e1, e2)
        det = _dot(e1, c23)
        q1, q2, q3 = _dot(e1, e1), _dot(e2, e2), _dot(e3, e3)
        off = tuple((q1 * c23[i] + q2 * c31[i] + q3 * c12[i]) / (2 * det) for i in range(3))
    return tuple(a[i] + off[i] for i in range(3)), _dot(off, off)


# ---- records -------------------------------------------------------------------------------
def _event_record(rank: int, interior: list[int], support: list[int], center, level, keff: int) -> dict:
    birth = rank if rank <= keff else None
    saddle = rank - 1 if 2 <= rank <= keff + 1 else None
    roles = []
    if saddle is not None:
        roles.append({"schema_version": SCHEMA_VERSION, "order": saddle, "morse_index": 1,
                      "local_multiplicity": comb(len(support) - 1, 1), "arm_count": len(support)})
    if birth is not None:
        roles.append({"schema_version": SCHEMA_VERSION, "order": birth, "morse_index": 0, "local_multiplicity": 1,
                      "arm_count": 0})
    roles.sort(key=lambda r: r["order"])
    witness = exact_rational3(center)
    lev = exact_level(level)
    projection = {"interior_ids": interior, "shell_ids": support, "minimal_support_ids": support,
                  "center_witness_homogeneous": witness, "squared_level_exact": lev}
    return {"schema_version": SCHEMA_VERSION, "event_id": canonical_id("CriticalEvent", projection),
            "closed_rank": rank, "interior_ids": interior, "shell_ids": support, "minimal_support_ids": support,
            "center_witness_homogeneous": witness, "squared_level_exact": lev,
            "barycentric_signs": [1] * len(support), "birth_order": birth, "saddle_order": saddle,
            "morse_roles": roles, "degeneracy_class": "general_position", "predicate_status": "certified_exact"}


def _zeros(names):
    return {k: 0 for k in names}


def build_contract(points: np.ndarray, source_index: np.ndarray, K: int, hier: Mapping[str, Any], *,
                   backend: str = "cuda_g4", run_id: str | None = None,
                   environment: Mapping[str, Any] | None = None) -> dict:
    """MorseHGP3DResult for one direct-hierarchy result.

    points: canonical coordinates in PointId order (n, 3), binary64;
    source_index: input position of every PointId;
    hier: the arrays of ehgp.Context.hierarchy (events, journal_batches, roles,
    families, nodes, children, births, bindings, saddles, groups, roots, vertical)."""
    pts = np.asarray(points, dtype=np.float64)
    n = len(pts)
    keff = int(hier["k_eff"])
    smax = min(keff + 1, n)
    P = [tuple(Fraction(float(x)) for x in p) for p in pts]
    # input
    certified = [{"schema_version": SCHEMA_VERSION, "point_id": i, "source_indices": [int(source_index[i])],
                  "multiplicity": 1, "coordinate_bits": [binary64_bits(x) for x in pts[i]],
                  "coordinate_unit": COORDINATE_UNIT, "predicate_status": "finite_exact_dyadic"} for i in range(n)]
    input_sha = canonical_id("Input", [{k: p[k] for k in ("point_id", "source_indices", "multiplicity",
                                                             "coordinate_bits")} for p in certified])
    # critical catalogue: singletons, then facade events
    ev = hier["events"]
    single_ids = []
    catalog = []
    for p in range(n):
        r = _event_record(1, [], [p], P[p], Fraction(0), keff)
        single_ids.append(r["event_id"])
        catalog.append(r)
    ev_ids, ev_level, ev_points = [], [], []
    for r in ev:
        sup = [int(x) for x in r["support_ids"][: r["support_size"]]]
        inter = [int(x) for x in r["interior_ids"][: r["interior_count"]]]
        c, lv = exact_sphere(P, sup)
        rec = _event_record(int(r["closed_rank"]), inter, sup, c, lv, keff)
        catalog.append(rec)
        ev_ids.append(rec["event_id"])
        ev_level.append(lv)
        ev_points.append(sorted(inter + sup))
    catalog.sort(key=lambda x: x["event_id"])

    def level_of(le) -> Fraction:
        return Fraction(0) if int(le) == ABSENT else ev_level[int(le)]

    def proj_event(pj: int) -> str:
        return single_ids[pj] if pj < n else ev_ids[pj - n]

    # equal-level batches
    roles = hier["roles"]
    jb = hier["journal_batches"]
    batch_ids, batch_records = [], []
    for b in jb:
        lv = level_of(b["level_event"])
        eids = sorted({proj_event(int(q["projection"]))
                       for q in roles[int(b["role_offset"]): int(b["role_offset"] + b["role_count"])]})
        projection = {"order": int(b["order"]), "squared_level_exact": exact_level(lv), "event_ids": eids}
        bid = canonical_id("EqualLevelBatch", projection)
        batch_ids.append(bid)
        batch_records.append({"schema_version": SCHEMA_VERSION, "batch_id": bid, "order": int(b["order"]),
                              "squared_level_exact": exact_level(lv), "event_ids": eids, "gamma_coface_ids": [],
                              "hyperedge_ids": [], "attachment_ids": [], "pre_lot_components": [],
                              "post_lot_components": [], "coverage_deltas": [], "events_complete": True,
                              "attachments_complete": False, "batch_status": "partial"})
    # forest nodes in creation order (children precede parents)
    nodes, children = hier["nodes"], hier["children"]
    groups, saddles, families, births = hier["groups"], hier["saddles"], hier["families"], hier["births"]
    node_ids, node_events, node_cover, node_records = [], [], [], {}
    for i, nd in enumerate(nodes):
        k = int(nd["order"])
        kids = [int(c) for c in children[int(nd["child_offset"]): int(nd["child_offset"] + nd["child_count"])]]
        if int(nd["kind"]) == 0:  # order-one birth of a singleton
            p = int(births[int(nd["birth_record"])]["projection"])
            eids, cover, bidx = [single_ids[p]], {p}, int(births[int(nd["birth_record"])]["batch"])
        else:
            g = groups[int(nd["atomic_group"])]
            sad = saddles[int(g["saddle_offset"]): int(g["saddle_offset"] + g["saddle_count"])]
            evs = [int(families[int(s["family"])]["event"]) for s in sad]
            eids = sorted({ev_ids[e] for e in evs})
            cover = set()
            for e in evs:
                cover.update(ev_points[e])
            for c in kids:
                cover.update(node_cover[c])
            bidx = int(g["batch"])
        kind = "birth" if int(nd["kind"]) in (0, 1) else "merge"
        lv = exact_level(level_of(nd["level_event"]))
        child_ids = sorted(node_ids[c] for c in kids)
        projection = {"order": k, "kind": kind, "squared_level": lv, "child_ids": child_ids,
                      "covered_point_ids": sorted(cover), "event_ids": eids}
        nid = canonical_id("MergeNode", projection)
        node_ids.append(nid)
        node_events.append(eids)
        node_cover.append(cover)
        node_records.setdefault(k, []).append(
            {"schema_version": SCHEMA_VERSION, "node_id": nid, "kind": kind, "squared_level": lv,
             "child_ids": child_ids, "covered_point_ids": sorted(cover), "event_ids": eids,
             "batch_id": batch_ids[bidx]})
    roots_by_order: dict[int, list[str]] = {}
    for r in hier["roots"]:
        roots_by_order.setdefault(int(r["order"]), []).append(node_ids[int(r["node"])])
    forests = []
    for k in range(1, keff + 1):
        recs = sorted(node_records.get(k, []), key=lambda x: x["node_id"])
        roots = sorted(roots_by_order.get(k, []))
        projection = {"order": k, "profile": "hgp_reduced", "forest_semantics": "partial_refinement",
                      "node_ids": [x["node_id"] for x in recs], "root_ids": roots, "coverage_log": []}
        forests.append({"schema_version": SCHEMA_VERSION, "forest_id": canonical_id("MergeForest", projection),
                        "order": k, "profile": "hgp_reduced", "forest_semantics": "partial_refinement",
                        "nodes": recs, "root_ids": roots, "coverage_log": [], "complete": False})
    # vertical maps
    by_source: dict[int, list[dict]] = {}
    for v in hier["vertical"]:
        s, t = int(v["source_node"]), int(v["target_node"])
        by_source.setdefault(int(v["source_order"]), []).append(
            {"schema_version": SCHEMA_VERSION, "source_node_id": node_ids[s], "target_node_id": node_ids[t],
             "at_squared_level": exact_level(level_of(nodes[s]["level_event"])), "method": "forest_propagation",
             "proof_reference_ids": node_events[s]})
    vertical_maps = []
    for k in range(2, keff + 1):
        assignments = sorted(by_source.get(k, []), key=lambda a: a["source_node_id"])
        projection = {"source_order": k, "target_order": k - 1, "assignments": assignments}
        vertical_maps.append({"schema_version": SCHEMA_VERSION, "map_id": canonical_id("VerticalMap", projection),
                              "source_order": k, "target_order": k - 1, "assignments": assignments,
                              "complete": True, "naturality_squares_checked": 0, "naturality_failures": 0})
    # run certificate
    env = {"git_commit": "0" * 40, "compiler": "nvcc", "compiler_version": "12.9", "cuda_version": "12.9",
           "driver_version": None, "hardware": "B200", "build_options_sha256": "0" * 64}
    if environment:
        env.update(environment)
    if run_id is None:
        run_id = canonical_id("Run", {"input_sha256": input_sha, "k_max": K, "backend": backend})
    snapshot_projection = {"boundary": "final", "sequence_number": 0}
    certificate = {
        "schema_version": SCHEMA_VERSION, "run_id": run_id, "reconstruction_contract_id": "hgp-reduced-v2",
        "proof_basis": "m1_conditional_contract", "result_kind": "partial_hierarchy",
        "requested_backend": backend, "effective_backend": backend, "requested_profile": "hgp_reduced",
        "effective_profile": "hgp_reduced", "requested_mode": "certified", "require_exact": False,
        "public_status": "conditional", "forest_semantics": "partial_refinement",
        "input_semantics": {
            "schema_version": SCHEMA_VERSION, "coordinate_encoding": "ieee754_binary64_bits",
            "coordinate_unit": COORDINATE_UNIT, "squared_level_unit": SQUARED_LEVEL_UNIT,
            "point_indexing": "zero_based",
            "canonical_point_order": "lexicographic_binary64_total_order_then_source_index",
            "non_finite_policy": "reject", "duplicate_policy": "reject",
            "signed_zero_policy": "canonicalize_to_positive_zero", "perturbation_policy": "none",
            "input_sha256": input_sha,
            "similarity_transform": {"schema_version": SCHEMA_VERSION, "applied": False,
                                     "scale": {"schema_version": SCHEMA_VERSION, "numerator": "1",
                                               "denominator": "1"},
                                     "translation": exact_rational3([Fraction(0)] * 3)}},
        "input_point_count": n, "k_max": K, "k_eff": keff, "s_max": smax, "m_star": max(smax - 2, 0),
        "general_position_status": "verified_relevant", "relevant_gp_complete": True,
        "canonical_children_complete": True, "active_cross_incidences_complete": False,
        "catalog_complete_by_rank": [True] * smax, "attachments_complete_by_order": [False] * keff,
        "gamma_complete_by_order": [False] * keff, "batches_complete_by_order": [True] * keff,
        "vertical_maps_complete": True, "partial_guarantees": ["partial_forest_refines_exact", "verified_events"],
        "exact_predicate_counts": _zeros(("fp32_proposals", "fp64_filtered_certified", "expansion_certified",
                                          "cpu_multiprecision_certified", "exact_zeros", "remaining_unknown")),
        "fallback_counts": _zeros(("gpu_to_cpu", "multiprecision", "overflow_queue", "unsupported_degeneracies",
                                   "numeric_failures")),
        "work_and_memory_counters": {**_zeros(("rejected_events", "canonical_cells_closed", "gamma_cofaces_emitted",
                                               "hyperedges_emitted", "external_runs", "bytes_read",
                                               "bytes_written", "peak_device_bytes", "peak_host_bytes",
                                               "peak_scratch_bytes", "output_bytes")),
                                     "candidate_events": len(catalog), "accepted_events": len(catalog)},
        "budget_policy": {"schema_version": SCHEMA_VERSION, "mode": "certified", "require_exact": False,
                          "byte_unit": "byte", "time_unit": "second", "device_budget_bytes": None,
                          "host_budget_bytes": None, "scratch_budget_bytes": None, "output_budget_bytes": None,
                          "time_budget_s": None, "stop_policy": "fail_closed"},
        "final_budget_snapshot": {
            "schema_version": SCHEMA_VERSION, "snapshot_id": canonical_id("BudgetSnapshot", snapshot_projection),
            "boundary": "final", "sequence_number": 0, "byte_unit": "byte", "time_unit": "second",
            "device_limit_bytes": None, "device_used_bytes": 0, "device_reserved_bytes": 0,
            "device_remaining_bytes": None, "host_limit_bytes": None, "host_used_bytes": 0,
            "host_reserved_bytes": 0, "host_remaining_bytes": None, "scratch_limit_bytes": None,
            "scratch_used_bytes": 0, "scratch_reserved_bytes": 0, "scratch_remaining_bytes": None,
            "output_limit_bytes": None, "output_used_bytes": 0, "output_reserved_bytes": 0,
            "output_remaining_bytes": None, "time_limit_s": None, "elapsed_s": 0.0, "remaining_s": None,
            "first_refusal_reason": None},
        "stop_reason": "completed", "unresolved_locus_ids": [], "software_environment": env,
    }
    certificate["certificate_id"] = canonical_id("RunCertificate", certificate)
    partial_scope = {"schema_version": SCHEMA_VERSION, "closed_parent_depths": [],
                     "closed_orders": list(range(1, keff + 1)), "catalog_complete_ranks": list(range(1, smax + 1)),
                     "canonical_cell_certificates": [], "verified_event_ids": sorted(x["event_id"] for x in catalog),
                     "unresolved_loci": [], "positive_guarantees": ["partial_forest_refines_exact",
                                                                    "verified_events"],
                     "absence_assertions_allowed": False}
    doc = {
        "schema_version": SCHEMA_VERSION, "run_id": run_id, "result_kind": "partial_hierarchy", "backend": backend,
        "profile": "hgp_reduced", "mode": "certified", "forest_semantics": "partial_refinement", "k_eff": keff,
        "critical_catalog": catalog, "gamma_cofaces": [], "gabriel_hyperedges": [], "attachments": [],
        "equal_level_batches": sorted(batch_records, key=lambda x: x["batch_id"]), "forests": forests,
        "vertical_maps": vertical_maps, "coverage_log": [], "materialized_point_sets": [],
        "partial_scope": partial_scope, "run_certificate": certificate,
    }
    doc["result_id"] = canonical_id("MorseHGP3DResult", {k: v for k, v in doc.items() if k != "run_certificate"})
    return doc


def dumps(doc: Mapping[str, Any]) -> str:
    """Canonical JSON text of a contract document."""
    return canonical_json(doc)
