"""Generates the LBVH golden fixtures in this directory from the reference's
own CPU code (oracle/_ref/libehgp_ref.so: CanonicalPointCloud::rejecting_duplicates
+ MortonLbvhIndex::build, compiled from morsehgp3d/src/cpu against the
project-written Boost shim).  Run here, where the reference tree exists:

    make -C oracle ref && python tests/golden/make_golden.py && python tests/golden/make_golden.py --geom
    python tests/golden/make_golden.py --pairs   # slow: the reference pair stream
    python tests/golden/make_golden.py --higher  # slow: the reference higher-support stream (n = 12)
    python tests/golden/make_golden.py --hierarchy  # slow: the reference direct chain up to the forest journal
    python tests/golden/make_golden.py --definition  # the Python exhaustive-Gamma hgp_reduced forests
    python tests/golden/make_golden.py --scale  # restatement digests at n = 216-256 (about 10 min)
    python tests/golden/make_golden.py --predicates  # the reference's predicate fixtures, answered by its replay tool
    python tests/golden/make_golden.py --scale-higher  # restatement triple/quad digests at n = 1000 (about 1.5 h)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "e-hgp_b200")]

from oracle import pyoracle  # noqa: E402
import workloads  # noqa: E402

TINY = np.nextafter(0.0, 1.0)
BIG = np.finfo(np.float64).max


def cases():
    yield "uniform256_s0", workloads.uniform_cube(256, 0)
    yield "uniform256_s1", workloads.uniform_cube(256, 1)
    yield "lattice5_f32", workloads.jittered_lattice(5, 3).astype(np.float64)
    # known-answer clouds of morsehgp3d/tests/unit/test_spatial_lbvh.cpp:641-744
    yield "collision4", np.array([[1, 1, 1], [2 * TINY, 0, 0], [0, 0, 0], [TINY, 0, 0]], float)
    yield "extrema4", np.array([[-BIG, -TINY, 0], [TINY, BIG, -BIG], [BIG, 0, TINY], [0, -BIG, BIG]], float)
    rng = np.random.Generator(np.random.PCG64(7))
    p = rng.random((600, 3))
    p[::3] = np.round(p[::3] * 7) / 7 + rng.random((200, 3)) * 1e-9  # many Morton collisions
    yield "collisions600", p
    q = rng.random((300, 3)) * 1e-300  # tiny exponents + a far point
    q[0] = [1e300, -1e300, 3.0]
    yield "spread300", q


def main():
    for name, pts in cases():
        r = pyoracle.lbvh_build(pts, "reference")
        np.savez_compressed(os.path.join(HERE, f"lbvh_{name}.npz"), points=pts,
                            **{k: r[k] for k in ("source_index", "leaves", "nodes", "counters", "root_aabb")},
                            root=np.uint64(r["root"]))
        print(name, len(pts), r["counters"])


if __name__ == "__main__" and len(sys.argv) == 1:
    main()


def geom_cases():
    yield "uniform64_s2", workloads.uniform_cube(64, 2)
    yield "lattice4_f32", workloads.jittered_lattice(4, 4).astype(np.float64)
    g = np.round(workloads.uniform_cube(120, 8) * 4) / 4 + 0.0  # quarter grid: many exact ties
    yield "grid120", np.unique(g, axis=0)


def frac(x):
    return [str(x.numerator), str(x.denominator)]


def main_geom():
    import json
    for name, pts in geom_cases():
        knn = pyoracle.knn(pts, 11, "reference")
        ef = pyoracle.emst_forest(pts, "reference")
        doc = {
            "points": pts.tolist(),
            "knn11": [[s, sh, frac(c)] for s, sh, c in knn],
            "edges": [[u, v, frac(d)] for u, v, d in ef["edges"]],
            "minima": [[r, l, s, u, v, frac(d)] for r, l, s, u, v, d in ef["minima"]],
            "accepted": [list(a) for a in ef["accepted"]],
            "levels": [frac(x) for x in ef["levels"]],
            "nodes": [list(nd) for nd in ef["nodes"]],
            "children": ef["children"],
            "batches": [list(b) for b in ef["batches"]],
            "root": ef["root"],
        }
        with open(os.path.join(HERE, f"geom_{name}.json"), "w") as f:
            json.dump(doc, f, separators=(",", ":"))
        print(name, len(pts), len(ef["nodes"]))


if __name__ == "__main__" and "--geom" in sys.argv:
    main_geom()


def parse_pairs(txt):
    """Records of ref_pairs / oracle_pairs text (see oracle/ref_driver.cpp)."""
    events, diags, status = [], [], None
    for line in txt.splitlines():
        head, _, tail = line.partition("|")
        t = head.split()
        if not t:
            continue
        ids = [int(x) for x in tail.split()]
        if t[0] == "P":
            events.append([int(t[1]), int(t[2]), int(t[3]), int(t[4]), t[5], t[6], t[7:11], ids])
        elif t[0] == "D":
            diags.append([int(x) for x in t[1:8]] + [t[8], t[9], t[10:14], ids])
        elif t[0] == "S":
            status = t[1]
    return {"events": events, "diagnostics": diags, "status": status}


def main_pairs():
    import json
    for name, pts in geom_cases():
        txt = pyoracle._text_call("ref_pairs", "reference", pts, 10)
        doc = {"points": pts.tolist(), "K": 10, **parse_pairs(txt)}
        with open(os.path.join(HERE, f"pairs_{name}.json"), "w") as f:
            json.dump(doc, f, separators=(",", ":"))
        print(name, len(pts), len(doc["events"]), len(doc["diagnostics"]), doc["status"], flush=True)


if __name__ == "__main__" and "--pairs" in sys.argv:
    main_pairs()


def higher_cases():
    yield "uniform12_s2", workloads.uniform_cube(12, 2)
    yield "lattice12", workloads.jittered_lattice(3, 6).astype(np.float64)[:12]
    # cube corners + face centres + centre: cospherical ties (extra-shell diagnostics)
    c = [[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)] + [[0.5, 0.5, 0.0], [0.5, 0.0, 0.5],
                                                                         [0.0, 0.5, 0.5], [0.5, 0.5, 0.5]]
    yield "cube12_ties", np.array(c, dtype=np.float64)


def parse_higher(txt):
    events, diags, status = [], [], None
    for line in txt.splitlines():
        head, _, tail = line.partition("|")
        t = head.split()
        if not t:
            continue
        ids = [int(x) for x in tail.split()]
        if t[0] in ("H", "G"):
            m = int(t[1])
            sup = [int(x) for x in t[2:2 + m]]
            rest = t[2 + m:]
            if t[0] == "H":
                events.append([m, sup, int(rest[0]), int(rest[1]), rest[2], rest[3], rest[4:8], ids])
            else:
                diags.append([m, sup] + [int(x) for x in rest[:5]] + [rest[5], rest[6], rest[7:11], ids])
        elif t[0] == "S":
            status = t[1]
    return {"events": events, "diagnostics": diags, "status": status}


def main_higher():
    import json
    for name, pts in higher_cases():
        txt = pyoracle._text_call("ref_higher", "reference", pts, 10)
        doc = {"points": pts.tolist(), "K": 10, **parse_higher(txt)}
        with open(os.path.join(HERE, f"higher_{name}.json"), "w") as f:
            json.dump(doc, f, separators=(",", ":"))
        print(name, len(pts), len(doc["events"]), len(doc["diagnostics"]), doc["status"], flush=True)


if __name__ == "__main__" and "--higher" in sys.argv:
    main_higher()


def hierarchy_cases():
    rng = np.random.Generator(np.random.PCG64(11))
    yield "uniform8_K10", rng.random((8, 3)), 10
    yield "uniform10_K10", rng.random((10, 3)), 10
    yield "uniform10_K3", rng.random((10, 3)), 3
    yield "lattice2_f32_K10", workloads.jittered_lattice(2, 5).astype(np.float64), 10
    # cube corners: every face and the whole cube are cospherical -> relevant extra shells
    yield "cube8_K10", np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float), 10


def main_hierarchy():
    import json
    for name, pts, K in hierarchy_cases():
        txt = pyoracle._text_call("ref_hierarchy", "reference", pts, K)
        doc = {"points": pts.tolist(), "K": K, "text": txt}
        with open(os.path.join(HERE, f"hier_{name}.json"), "w") as f:
            json.dump(doc, f, separators=(",", ":"))
        print(name, len(pts), len(txt.splitlines()), txt.splitlines()[-1], flush=True)


if __name__ == "__main__" and "--hierarchy" in sys.argv:
    main_hierarchy()


# ---- the normative hgp_reduced definition (Python exhaustive-Gamma oracle) ------------
# morsehgp3d_oracle (stdlib only) inside the reference checkout; run where the reference exists
REF_PY = os.path.join(pyoracle.reference_root() or "", "reference")


def definition_cases():
    rng = np.random.Generator(np.random.PCG64(29))
    yield "uniform6_K10", rng.random((6, 3)), 10
    yield "uniform7_K10", rng.random((7, 3)), 10
    yield "uniform8_K10", rng.random((8, 3)), 10
    yield "uniform8_K3", rng.random((8, 3)), 3
    yield "lattice2_f32_K10", workloads.jittered_lattice(2, 9).astype(np.float64), 10


def main_definition():
    """Forests of run_oracle(points, K, profile='hgp_reduced')
    (reference/morsehgp3d_oracle/oracle.py:211, hierarchy.py:309-498): per order the
    nodes in creation order as (kind, level numerator, level denominator, child indices
    within the order), and the final root indices."""
    import json
    sys.path.insert(0, REF_PY)
    from morsehgp3d_oracle.oracle import run_oracle
    for name, pts, K in definition_cases():
        res = run_oracle([tuple(float(x) for x in p) for p in pts], K, profile="hgp_reduced")
        forests = []
        for o in res.orders:
            f = o.forest
            index = {nd.node_id: i for i, nd in enumerate(f.nodes)}
            nodes = [[nd.kind, str(nd.squared_level.numerator), str(nd.squared_level.denominator),
                      [index[c] for c in nd.child_ids]] for nd in f.nodes]
            forests.append({"order": o.order, "nodes": nodes, "roots": sorted(index[r] for r in f.root_ids)})
        # vertical assignments as the contract serializer forms them
        # (reference/morsehgp3d_oracle/serialization.py:1040-1099): every source node maps, at
        # its own level on the closed cut, to the lower-order root whose component contains it
        vertical = []
        for fam in res.vertical_maps:
            src = res.for_order(fam.source_order).forest
            tgt = res.for_order(fam.target_order).forest
            sidx = {nd.node_id: i for i, nd in enumerate(src.nodes)}
            tidx = {nd.node_id: i for i, nd in enumerate(tgt.nodes)}
            closed = {mp.squared_level: mp for mp in fam.maps if mp.closed}
            for nd in src.nodes:
                comp = [c for c in src.cut(nd.squared_level, closed=True).components if c.root_id == nd.node_id]
                tf = closed[nd.squared_level].assignment_by_source[comp[0].facet_point_ids]
                cand = [c for c in tgt.cut(nd.squared_level, closed=True).components if c.facet_point_ids == tf]
                vertical.append([fam.source_order, sidx[nd.node_id], tidx[cand[0].root_id]])
        # the contract serializer's critical catalogue (serialization.py:723-793)
        from morsehgp3d_oracle.serialization import serialize_oracle_result
        catalog = serialize_oracle_result(res, run_id="0" * 64)["critical_catalog"]
        doc = {"points": pts.tolist(), "K": K, "k_eff": res.k_eff, "forests": forests, "vertical": vertical,
               "catalog": catalog}
        with open(os.path.join(HERE, f"definition_{name}.json"), "w") as fh:
            json.dump(doc, fh, separators=(",", ":"))
        print(name, len(pts), [len(f["nodes"]) for f in forests], flush=True)


if __name__ == "__main__" and "--definition" in sys.argv:
    main_definition()


# ---- parity at scale: digests of the restatement's supports and hierarchy ----------------
def scale_cases():
    """cfg1 (256 i.i.d. uniform points, seeds 0-9), a 6^3 jittered lattice, and 256-point
    samples of the clustered generator with and without the 2^-10 snapping, K = 10."""
    for seed in range(10):
        yield f"uniform256_s{seed}", workloads.uniform_cube(256, seed)
    yield "lattice6_f32", workloads.jittered_lattice(6, 5).astype(np.float64)
    for seed in range(3):
        yield f"clustered256_snap_s{seed}", workloads.clustered(256, 100 + seed)
    for seed in range(2):
        yield f"clustered256_s{seed}", workloads.clustered(256, 200 + seed, snapped=0.0)


def higher_digest(rec: dict) -> str:
    """Digest of higher-support records in the parsed form (pyoracle.parse_higher and
    tests/geomcheck.gpu_higher_records give the same tuples)."""
    import hashlib
    return hashlib.sha256(repr((rec["events"], rec["diagnostics"])).encode()).hexdigest()


def text_digest(text: str) -> str:
    import hashlib
    return hashlib.sha256(text.encode()).hexdigest()


def _scale_one(args):
    name, pts, K = args
    P = np.asarray(pts, np.float64)
    snap = pyoracle.lbvh_build(P)
    canon = P[snap["source_index"].astype(np.int64)]
    hi = pyoracle.higher(canon, K)
    txt = pyoracle.hierarchy(P, K)
    lines = txt.splitlines()
    return name, {"points": P.tolist(), "K": K, "higher_sha256": higher_digest(hi),
                  "higher_events": len(hi["events"]), "higher_diagnostics": len(hi["diagnostics"]),
                  "hierarchy_sha256": text_digest(txt), "hierarchy_lines": len(lines),
                  "hierarchy_last": lines[-1], "refused": txt.rstrip().endswith("D 4 3 4"),
                  "facade_events": sum(1 for l in lines if l.startswith("F ")),
                  "diagnostics": next(int(l.split()[1]) for l in lines if l.startswith("X "))}


def main_scale():
    import json
    import multiprocessing as mp
    jobs = [(name, pts, 10) for name, pts in scale_cases()]
    out = {}
    with mp.get_context("spawn").Pool(4) as pool:
        for name, d in pool.imap_unordered(_scale_one, jobs):
            out[name] = d
            print(name, d["higher_events"], d["higher_diagnostics"], d["hierarchy_lines"], d["hierarchy_last"],
                  flush=True)
    with open(os.path.join(HERE, "scale_digests.json"), "w") as fh:
        json.dump({k: out[k] for k, _, _ in jobs}, fh, separators=(",", ":"))


if __name__ == "__main__" and "--scale" in sys.argv:
    main_scale()


# ---- the reference's predicate fixtures, answered by its own replay tool ---------------
PRED_KINDS = ("support_sphere_side", "compare_support_levels", "circumcenter_support_analysis",
              "binary64_circumcenter_support_analysis", "compare_squared_distances")


def main_predicates():
    """Every fixture of morsehgp3d/tests/fixtures/predicates/ whose predicate this path
    evaluates, with the answer of the reference's own tool (oracle/_ref/replay_predicate,
    morsehgp3d/src/tools/predicate_replay.cpp compiled unmodified)."""
    import glob
    import json
    import subprocess
    root = pyoracle.reference_root()
    tool = os.path.join(ROOT, "oracle", "_ref", "replay_predicate")
    out = []
    for path in sorted(glob.glob(os.path.join(root, "morsehgp3d", "tests", "fixtures", "predicates", "*.json"))):
        d = json.load(open(path))
        kind = d.get("predicate")
        if kind not in PRED_KINDS:
            continue
        if kind == "support_sphere_side":
            groups = {"support": d["support"], "point": [d["point"]]}
            args = [str(len(d["support"]))] + [w for p in d["support"] for w in p] + d["point"]
        elif kind == "compare_support_levels":
            groups = {"left": d["left_support"], "right": d["right_support"]}
            args = ([str(len(d["left_support"]))] + [w for p in d["left_support"] for w in p] +
                    [str(len(d["right_support"]))] + [w for p in d["right_support"] for w in p])
        elif kind == "compare_squared_distances":
            groups = {"points": d["points"]}
            args = [w for p in d["points"] for w in p]
        else:
            groups = {"points": d["points"]}
            args = [str(len(d["points"]))] + [w for p in d["points"] for w in p]
        r = subprocess.run([tool, kind, *args], capture_output=True, text=True)
        res = json.loads(r.stdout) if r.returncode == 0 and r.stdout.strip() else {"error": r.stderr.strip()}
        keep = {k: res[k] for k in ("sign", "support_status", "support_kind", "classification", "ordering",
                                    "certification_stage", "error") if k in res}
        out.append({"fixture": os.path.basename(path), "predicate": kind, "groups": groups, "reference": keep})
        print(os.path.basename(path), kind, keep, flush=True)
    with open(os.path.join(HERE, "predicates_ref.json"), "w") as fh:
        json.dump(out, fh, indent=0, sort_keys=True)


if __name__ == "__main__" and "--predicates" in sys.argv:
    main_predicates()


# ---- completeness beyond the plain workload's size (triple/quad records only) -----------
def main_scale_higher():
    """Digests of the restatement's complete triple/quad stream (brute force over every
    tuple, FP64-filtered, exact where undecided) for 1,000-point clouds: i.i.d. uniform and a
    10^3 jittered lattice.  About 45 minutes each on 8 host threads."""
    import json
    cases = [("uniform1000_s0", workloads.uniform_cube(1000, 0)),
             ("lattice10_f32", workloads.jittered_lattice(10, 6).astype(np.float64))]
    out = {}
    for name, pts in cases:
        snap = pyoracle.lbvh_build(pts)
        canon = pts[snap["source_index"].astype(np.int64)]
        hi = pyoracle.higher(canon, 10)
        out[name] = {"points": pts.tolist(), "K": 10, "higher_sha256": higher_digest(hi),
                     "higher_events": len(hi["events"]), "higher_diagnostics": len(hi["diagnostics"])}
        print(name, out[name]["higher_events"], out[name]["higher_diagnostics"], flush=True)
        with open(os.path.join(HERE, "scale_higher_digests.json"), "w") as fh:
            json.dump(out, fh, separators=(",", ":"))


if __name__ == "__main__" and "--scale-higher" in sys.argv:
    main_scale_higher()
