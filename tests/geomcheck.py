"""Helpers shared by the k-NN / EMST / k=1 forest tests: conversion of the
CUDA path's outputs and of golden fixtures to the oracle's text-record form."""
from fractions import Fraction
import json

import numpy as np

import ehgp


def load_golden(path):
    d = json.load(open(path))
    F = lambda x: Fraction(int(x[0]), int(x[1]))
    return {
        "points": np.array(d["points"], dtype=np.float64),
        "knn11": [(s, sh, F(c)) for s, sh, c in d["knn11"]],
        "emst": {
            "edges": [(u, v, F(x)) for u, v, x in d["edges"]],
            "minima": [(r, l, s, u, v, F(x)) for r, l, s, u, v, x in d["minima"]],
            "accepted": [tuple(a) for a in d["accepted"]],
            "levels": [F(x) for x in d["levels"]],
            "nodes": [tuple(n) for n in d["nodes"]],
            "children": d["children"],
            "batches": [tuple(b) for b in d["batches"]],
            "root": d["root"],
        },
    }


def gpu_knn_records(ctx, k):
    """ehgp_knn output as (strict ids, first shell ids, shell size, cutoff) per PointId."""
    r = ctx.knn(k)
    out = []
    for p in range(len(r["ids"])):
        strict, shell = (int(x) for x in r["meta"][p])
        ids = [int(x) for x in r["ids"][p]]
        out.append((ids[:strict], ids[strict:], shell, r["cutoff"][p]))
    return out


def knn_matches(gpu, ref, k):
    """gpu: gpu_knn_records; ref: oracle (strict, shell, cutoff) list."""
    assert len(gpu) == len(ref)
    for p, ((gs, gsh, gshell, gc), (rs, rsh, rc)) in enumerate(zip(gpu, ref)):
        assert gs == rs, (p, gs, rs)
        assert gsh == rsh[: k - len(rs)], (p, gsh, rsh)
        assert gshell == len(rsh), (p, gshell, len(rsh))
        assert gc == rc, (p, gc, rc)


def gpu_emst_forest(ctx):
    """ehgp_emst + ehgp_k1_forest in the oracle's record form."""
    S, valid = ctx.scale()
    assert valid
    den = 1 << (2 * S)
    e = ctx.emst()
    D = [ehgp.limbs_to_int(x) for x in e["D"]]
    edges = [(int(u), int(v), Fraction(d, den)) for u, v, d in zip(e["u"], e["v"], D)]

    def d2(a, b):
        return None  # squared lengths of minima come from the edge list

    lengths = {(u, v): x for u, v, x in edges}
    minima, accepted = [], []
    for rnd, label, src, tgt in (tuple(int(x) for x in m) for m in e["minima"]):
        u, v = min(src, tgt), max(src, tgt)
        minima.append((rnd, label, src, u, v, lengths.get((u, v))))
    minima.sort()
    by_round = {}
    for rnd, _, _, u, v, x in minima:
        by_round.setdefault(rnd, set()).add((x, u, v))
    for rnd in sorted(by_round):
        for x, u, v in sorted(by_round[rnd]):
            accepted.append((rnd, u, v))
    f = ctx.k1_forest()
    levels = [Fraction(ehgp.limbs_to_int(x), den) / 4 for x in f["level_num"]]
    return {
        "edges": edges, "minima": minima, "accepted": accepted, "levels": levels,
        "nodes": [tuple(int(x) for x in nd) for nd in f["nodes"]],
        "children": [int(x) for x in f["children"]],
        "batches": [tuple(int(x) for x in b) for b in f["batches"]],
        "root": f["root"], "rounds": e["rounds"],
    }


def emst_forest_matches(gpu, ref):
    for key in ("edges", "minima", "accepted", "levels", "nodes", "children", "batches", "root"):
        assert gpu[key] == ref[key], key


def load_golden_pairs(path):
    """pairs_*.json (tests/golden/make_golden.py --pairs) -> oracle record tuples."""
    d = json.load(open(path))
    F = lambda a, b: Fraction(int(a), int(b))
    ev = [(u, v, r, ext, F(ln, ld), tuple(F(c, cen[3]) for c in cen[:3]), tuple(ids))
          for u, v, r, ext, ln, ld, cen, ids in d["events"]]
    dg = [(u, v, sh, w, mr, orr, ext, F(ln, ld), tuple(F(c, cen[3]) for c in cen[:3]), tuple(ids))
          for u, v, sh, w, mr, orr, ext, ln, ld, cen, ids in d["diagnostics"]]
    return np.array(d["points"], dtype=np.float64), d["K"], {"events": ev, "diagnostics": dg, "status": d["status"]}


def gpu_pair_records(ctx, K, points_canonical):
    """ehgp_pairs output converted to the oracle's (events, diagnostics) tuples.

    points_canonical: binary64 coordinates in PointId order (for the exact centre)."""
    S, valid = ctx.scale()
    assert valid
    n = len(points_canonical)
    r = ctx.pairs(K)
    ev, dg = [], []
    for rec, lv in zip(r["records"], r["level_num"]):
        u, v = int(rec["u"]), int(rec["v"])
        I, sh = int(rec["interior_count"]), int(rec["shell_count"])
        level = Fraction(ehgp.limbs_to_int(lv), 1 << (2 * S)) / 4
        center = tuple((Fraction(float(points_canonical[u][a])) + Fraction(float(points_canonical[v][a]))) / 2
                       for a in range(3))
        ids = tuple(int(x) for x in rec["interior_ids"][:I])
        if sh == 2:
            ev.append((u, v, I + 2, n - I - 2, level, center, ids))
        else:
            dg.append((u, v, sh, int(rec["extra_shell_witness"]), I + 2, I + sh, n - I - sh, level, center, ids))
    return {"events": ev, "diagnostics": dg, "status": "complete"}


def pairs_match(gpu, ref):
    for key in ("events", "diagnostics"):
        g, r = gpu[key], ref[key]
        if g != r:
            gs, rs = set(g), set(r)
            raise AssertionError(f"{key}: {len(g)} vs {len(r)}; only gpu {sorted(gs - rs)[:3]}; "
                                 f"only oracle {sorted(rs - gs)[:3]}")
    assert ref["status"] == "complete"


def exact_sphere(P, ids):
    """Exact circumcentre and squared level of a 3- or 4-point support (Fractions)."""
    pts = [[Fraction(float(x)) for x in P[i]] for i in ids]
    a = pts[0]
    e = [[p[k] - a[k] for k in range(3)] for p in pts[1:]]
    dot = lambda u, v: sum(x * y for x, y in zip(u, v))
    cross = lambda u, v: [u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]]
    if len(ids) == 3:
        G11, G12, G22 = dot(e[0], e[0]), dot(e[0], e[1]), dot(e[1], e[1])
        A = G11 * G22 - G12 * G12
        N = [G22 * (G11 - G12) * e[0][k] + G11 * (G22 - G12) * e[1][k] for k in range(3)]
    else:
        c23, c31, c12 = cross(e[1], e[2]), cross(e[2], e[0]), cross(e[0], e[1])
        A = dot(e[0], c23)
        N = [dot(e[0], e[0]) * c23[k] + dot(e[1], e[1]) * c31[k] + dot(e[2], e[2]) * c12[k] for k in range(3)]
    off = [x / (2 * A) for x in N]
    return tuple(a[k] + off[k] for k in range(3)), dot(off, off)


def gpu_higher_records(ctx, K, points_canonical):
    """ehgp_higher output converted to the oracle's (events, diagnostics) tuples."""
    n = len(points_canonical)
    ev, dg = [], []
    for r in ctx.higher(K):
        m = int(r["size"])
        ids = tuple(int(x) for x in r["ids"][:m])
        I, sh = int(r["interior_count"]), int(r["shell_count"])
        center, level = exact_sphere(points_canonical, ids)
        iids = tuple(int(x) for x in r["interior_ids"][:I])
        if sh == m:
            ev.append((m, ids, I + m, n - I - m, level, center, iids))
        else:
            dg.append((m, ids, sh, int(r["extra_shell_witness"]), I + m, I + sh, n - I - sh, level, center, iids))
    return {"events": ev, "diagnostics": dg, "status": "complete"}


def higher_match(gpu, ref):
    for key in ("events", "diagnostics"):
        g, r = gpu[key], ref[key]
        if g != r:
            gs, rs = set(g), set(r)
            raise AssertionError(f"{key}: {len(g)} vs {len(r)}; only gpu {sorted(gs - rs)[:2]}; "
                                 f"only oracle {sorted(rs - gs)[:2]}")


# ---- direct hierarchy ------------------------------------------------------------
def _frac_text(f: Fraction) -> str:
    return f"{f.numerator} {f.denominator}"


def gpu_hierarchy_text(ctx, K, res=None) -> str:
    """Renders an ehgp_hierarchy result in the line format of the oracle and of the
    reference driver (oracle/ref_driver.cpp ref_hierarchy)."""
    A = ehgp.ABSENT
    if res is None:
        res = ctx.hierarchy(K)
    n = ctx.n
    keff = int(res["k_eff"])
    ev = res["events"]
    lev_cache = {}

    def level(e):
        if e == A:
            return "0 1"
        if e not in lev_cache:
            lev_cache[e] = _frac_text(ctx.event_level(int(e)))
        return lev_cache[e]

    def opt(x):
        return "-" if x == A else str(int(x))

    def facet(proj):
        if proj < n:
            return [int(proj)]
        r = ev[proj - n]
        f = [int(x) for x in r["interior_ids"][: r["interior_count"]]] + \
            [int(x) for x in r["support_ids"][: r["support_size"]]]
        return sorted(f)

    def key(f):
        return " ".join([str(len(f))] + [str(x) for x in f])

    out = []
    for i, r in enumerate(ev):
        rank = int(r["closed_rank"])
        ids = " ".join(str(int(x)) for x in r["support_ids"][: r["support_size"]])
        inter = "".join(" " + str(int(x)) for x in r["interior_ids"][: r["interior_count"]])
        birth = str(rank) if rank <= keff else "-"
        saddle = str(rank - 1) if 2 <= rank <= keff + 1 else "-"
        out.append(f"F {i} {int(r['support_size'])} {ids} |{inter} | {rank} {n - rank} {level(i)} {birth} {saddle}")
    out.append(f"X {int(res['diagnostics'])}")
    for i, b in enumerate(res["journal_batches"]):
        out.append(f"J {i} {int(b['order'])} {level(b['level_event'])} {int(b['role_offset'])} {int(b['role_count'])} "
                   f"{int(b['birth_roles'])} {int(b['saddle_roles'])}")
    for i, q in enumerate(res["roles"]):
        out.append(f"Q {i} {int(q['batch'])} {int(q['projection'])} {int(q['role'])}")
    fam_of_seed = {}
    for i, f in enumerate(res["families"]):
        b = res["journal_batches"][f["batch"]]
        out.append(f"Y {i} {int(f['event'])} {int(f['projection'])} {int(f['role_record'])} {int(f['batch'])} "
                   f"{int(f['order'])} {level(b['level_event'])} {int(f['arm_offset'])} {int(f['arm_count'])}")
        for s in range(int(f["arm_offset"]), int(f["arm_offset"] + f["arm_count"])):
            fam_of_seed[s] = i
    for s, u in enumerate(res["arm_removed"]):
        out.append(f"Z {s} {fam_of_seed[s]} {int(u)}")
    for i, nd in enumerate(res["nodes"]):
        out.append(f"N {i} {int(nd['order'])} {level(nd['level_event'])} {int(nd['kind'])} {int(nd['child_offset'])} "
                   f"{int(nd['child_count'])} {opt(nd['birth_record'])} {opt(nd['atomic_group'])}")
    out.append("C" + "".join(" " + str(int(c)) for c in res["children"]))
    for i, bt in enumerate(res["births"]):
        out.append(f"B {i} {int(bt['projection'])} {int(bt['batch'])} {int(bt['order'])} {int(bt['handle'])} "
                   f"{opt(bt['order_one_node'])} | {key(facet(int(bt['projection'])))}")
    fams = res["families"]
    for i, a in enumerate(res["bindings"]):
        f = fams[a["family"]]
        removed = int(res["arm_removed"][a["arm_seed"]])
        arm = [x for x in facet(int(f["projection"])) if x != removed]
        out.append(f"A {i} {int(a['arm_seed'])} {int(a['family'])} {int(a['carrier'])} {opt(a['prior_root'])} | "
                   f"{key(arm)}")
    for i, s in enumerate(res["saddles"]):
        out.append("S " + " ".join(str(int(x)) for x in [i] + [s[f] for f in ehgp.FOREST_SADDLE.names]))
    for i, g in enumerate(res["groups"]):
        vals = [int(g[f]) for f in ehgp.FOREST_GROUP.names]
        vals[8] = opt(vals[8])
        out.append("G " + " ".join(str(x) for x in [i] + vals))
    for i, b in enumerate(res["batches"]):
        out.append(f"T {i} {i} {int(b['order'])} {level(b['level_event'])} " +
                   " ".join(str(int(b[f])) for f in ehgp.FOREST_BATCH.names[2:]))
    for i, r in enumerate(res["roots"]):
        out.append(f"R {i} {int(r['order'])} {int(r['handle'])} {int(r['node'])}")
    out.append("D 5 5 13")
    return "\n".join(out) + "\n"


def hierarchy_diff(a: str, b: str) -> str:
    """First differing line of two hierarchy texts ('' when equal)."""
    la, lb = a.splitlines(), b.splitlines()
    for x, y in zip(la, lb):
        if x != y:
            return f"gpu: {x[:240]}\nref: {y[:240]}"
    if len(la) != len(lb):
        return f"line counts {len(la)} vs {len(lb)}"
    return ""


# ---- the normative hgp_reduced definition ------------------------------------------
def forests_from_hier_text(text: str) -> list[dict]:
    """Per-order forests (the definition's layout) from a direct-hierarchy text:
    nodes of each order in creation order as [kind, num, den, child indices within
    the order] (order-one and reduced births are 'birth', multifusions 'merge'), and
    the final roots as indices within the order."""
    nodes, children, roots = [], [], []
    for line in text.splitlines():
        f = line.split()
        if not f:
            continue
        if f[0] == "N":
            nodes.append((int(f[1]), int(f[2]), f[3], f[4], int(f[5]), int(f[6]), int(f[7])))
        elif f[0] == "C":
            children = [int(x) for x in f[1:]]
        elif f[0] == "R":
            roots.append((int(f[2]), int(f[4])))
    orders = sorted({nd[1] for nd in nodes} | {o for o, _ in roots})
    out = []
    for k in orders:
        ids = [nd[0] for nd in nodes if nd[1] == k]
        local = {g: i for i, g in enumerate(ids)}
        fn = []
        for nd in nodes:
            if nd[1] != k:
                continue
            _, _, num, den, kind, off, cnt = nd
            fn.append(["birth" if kind in (0, 1) else "merge", num, den, [local[c] for c in children[off:off + cnt]]])
        out.append({"order": k, "nodes": fn, "roots": sorted(local[g] for o, g in roots if o == k)})
    return out


def definition_match(ours: list[dict], golden: list[dict]) -> str:
    """'' when every order of the golden definition forest equals ours (orders with no
    node on either side compare equal)."""
    by = {f["order"]: f for f in ours}
    for g in golden:
        o = by.get(g["order"], {"nodes": [], "roots": []})
        if o["nodes"] != g["nodes"]:
            return f"order {g['order']}: nodes differ\n ours {o['nodes'][:6]}\n def  {g['nodes'][:6]}"
        if o["roots"] != g["roots"]:
            return f"order {g['order']}: roots {o['roots']} vs {g['roots']}"
    return ""


def vertical_from_hier_text(text: str) -> list[list[int]]:
    """Vertical assignments [source order, source index, target index] (indices within
    their orders) derived from a direct-hierarchy text: a reduced node N of order k at
    level a takes a carrier birth of its group; that birth's event is also a saddle of
    order k - 1, whose group's resulting root, climbed through multifusion parents whose
    level is <= a (closed cut), is the image of N."""
    from fractions import Fraction
    N, C, B, A, S, G, Y = [], [], [], [], [], [], []
    for line in text.splitlines():
        f = line.split()
        if not f:
            continue
        t = f[0]
        if t == "N":
            N.append((int(f[2]), Fraction(int(f[3]), int(f[4])), int(f[5]), int(f[6]), int(f[7]), f[9]))
        elif t == "C":
            C = [int(x) for x in f[1:]]
        elif t == "B":
            B.append(int(f[2]))  # projection, indexed by handle
        elif t == "A":
            A.append(int(f[4]))  # carrier
        elif t == "S":
            S.append((int(f[2]), int(f[5]), int(f[10])))  # family, arm offset, group
        elif t == "G":
            G.append(int(f[11]))  # resulting root node
        elif t == "Y":
            Y.append((int(f[2]), int(f[6])))  # event, order
    n = sum(1 for nd in N if nd[0] == 1 and nd[2] == 0)
    parent = {}
    for i, nd in enumerate(N):
        if nd[2] == 2:
            for c in C[nd[3]:nd[3] + nd[4]]:
                parent[c] = i
    fam_of = {(ev, order): fi for fi, (ev, order) in enumerate(Y)}
    sad_of_fam = {s[0]: si for si, s in enumerate(S)}
    first_sad_of_group = {}
    for si, s in enumerate(S):
        first_sad_of_group.setdefault(s[2], si)
    local, counter = {}, {}
    for i, nd in enumerate(N):
        local[i] = counter.get(nd[0], 0)
        counter[nd[0]] = local[i] + 1
    out = []
    for i, nd in enumerate(N):
        k, lev, kind = nd[0], nd[1], nd[2]
        if k < 2:
            continue
        g = int(nd[5])
        carrier = A[S[first_sad_of_group[g]][1]]
        ev = B[carrier] - n
        R = G[S[sad_of_fam[fam_of[(ev, k - 1)]]][2]]
        while R in parent and N[parent[R]][1] <= lev:
            R = parent[R]
        out.append([k, local[i], local[R]])
    return out


def hier_dict_from_text(text: str, n: int, keff: int) -> dict:
    """The arrays of ehgp.Context.hierarchy rebuilt from a direct-hierarchy text
    (restatement or reference), vertical maps included (global node ids)."""
    from fractions import Fraction
    L = {t: [] for t in "FJQYZNBASGTR"}
    C = []
    for line in text.splitlines():
        f = line.split()
        if not f:
            continue
        if f[0] == "C":
            C = [int(x) for x in f[1:]]
        elif f[0] in L:
            L[f[0]].append(f)
    first_at = {}
    events = np.zeros(len(L["F"]), ehgp.EVENT_RECORD)
    for i, f in enumerate(L["F"]):
        size = int(f[2])
        sup = [int(x) for x in f[3:3 + size]]
        bar = f.index("|", 3 + size)
        bar2 = f.index("|", bar + 1)
        inter = [int(x) for x in f[bar + 1:bar2]]
        rank, num, den = int(f[bar2 + 1]), int(f[bar2 + 3]), int(f[bar2 + 4])
        events[i]["support_size"] = size
        events[i]["support_ids"][:size] = sup
        events[i]["interior_count"] = len(inter)
        events[i]["interior_ids"][:len(inter)] = inter
        events[i]["closed_rank"] = rank
        first_at.setdefault(Fraction(num, den), i)

    def lev(num, den):
        v = Fraction(int(num), int(den))
        return ehgp.ABSENT if v == 0 else first_at[v]

    def arr(rows, dtype):
        a = np.zeros(len(rows), dtype)
        for i, r in enumerate(rows):
            for name, v in zip(dtype.names, r):
                a[i][name] = ehgp.ABSENT if v == "-" else int(v)
        return a

    opt = lambda x: ehgp.ABSENT if x == "-" else int(x)
    jb = arr([(f[2], lev(f[3], f[4]), f[5], f[6], f[7], f[8]) for f in L["J"]], ehgp.JOURNAL_BATCH)
    roles = arr([(f[2], f[3], f[4]) for f in L["Q"]], ehgp.ROLE_RECORD)
    fams = arr([(f[2], f[3], f[4], f[5], f[6], f[9], f[10]) for f in L["Y"]], ehgp.FAMILY_RECORD)
    removed = np.array([int(f[3]) for f in L["Z"]], np.uint32)
    nodes = arr([(f[2], lev(f[3], f[4]), f[5], f[6], f[7], opt(f[8]), opt(f[9])) for f in L["N"]], ehgp.FOREST_NODE)
    births = arr([(f[2], f[3], f[4], f[5], opt(f[6])) for f in L["B"]], ehgp.FOREST_BIRTH)
    binds = arr([(f[2], f[3], f[4], opt(f[5])) for f in L["A"]], ehgp.FOREST_BINDING)
    sads = arr([f[2:11] for f in L["S"]], ehgp.FOREST_SADDLE)
    grps = arr([f[2:10] + [opt(f[10]), f[11], f[12]] for f in L["G"]], ehgp.FOREST_GROUP)
    fb = arr([(f[3], lev(f[4], f[5])) + tuple(f[6:16]) for f in L["T"]], ehgp.FOREST_BATCH)
    roots = arr([(f[2], f[3], f[4]) for f in L["R"]], ehgp.FOREST_ROOT)
    # vertical maps in global node ids
    order_start = {}
    for i, nd in enumerate(nodes):
        order_start.setdefault(int(nd["order"]), i)
    vert = []
    for k, si, ti in vertical_from_hier_text(text):
        s = order_start[k] + si
        vert.append((s, order_start[k - 1] + ti, k, int(nodes[s]["level_event"])))
    vertical = arr(sorted(vert), ehgp.VERTICAL_ASSIGNMENT)
    return {"k_eff": keff, "events": events, "journal_batches": jb, "roles": roles, "families": fams,
            "arm_removed": removed, "nodes": nodes, "children": np.array(C, np.uint32), "births": births,
            "bindings": binds, "saddles": sads, "groups": grps, "batches": fb, "roots": roots, "vertical": vertical}
