"""ORACLE loader — test infrastructure only (tests/, smoke() and bench.py's
CPU-baseline leg), never part of the product path.

Two independent CPU oracles, both driven through ctypes:
  * `restatement`: oracle/lib/libehgp_oracle.so, the project-written plain
    C++ restatement of the reference's algorithm (oracle/ehgp_oracle.cpp);
  * `reference`:   oracle/_ref/libehgp_ref.so, the reference's own CPU code
    (Ludwig-H/E-HGP morsehgp3d/src/cpu) compiled unmodified against the
    project-written Boost shim (oracle/Makefile + oracle/ref_driver.cpp).
Either may be absent (the reference tree is needed to build `_ref`); callers
check `available()`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
from fractions import Fraction

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT = os.path.join(HERE, "lib", "libehgp_oracle.so")
REFERENCE = os.path.join(HERE, "_ref", "libehgp_ref.so")

_libs: dict[str, C.CDLL] = {}
_ref_root: list[str | None] = []


def reference_root() -> str | None:
    """Root of the reference checkout (EHGP_REFERENCE_ROOT, else the default of this
    directory's Makefile, the recipe that compiles it), or None when it is absent."""
    if not _ref_root:
        root = os.environ.get("EHGP_REFERENCE_ROOT")
        if not root:
            import subprocess
            try:
                root = subprocess.run(["make", "-s", "-C", HERE, "print-ref-root"], capture_output=True, text=True,
                                      timeout=30).stdout.strip()
            except Exception:
                root = None
        _ref_root.append(root if root and os.path.isdir(root) else None)
    return _ref_root[0]


class OracleError(ValueError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def available(which: str) -> bool:
    return os.path.exists(RESTATEMENT if which == "restatement" else REFERENCE)


def _lib(which: str) -> C.CDLL:
    if which not in _libs:
        path = RESTATEMENT if which == "restatement" else REFERENCE
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing: run `make -C oracle`")
        _libs[which] = C.CDLL(path)
    return _libs[which]


def _p(a):
    return None if a is None else a.ctypes.data


def lbvh_build(points: np.ndarray, which: str = "restatement") -> dict:
    """Canonical cloud + Morton LBVH snapshot (same layout as the CUDA path)."""
    pts = np.ascontiguousarray(points, dtype=np.float64)
    n = pts.shape[0]
    out = {
        "source_index": np.empty(n, np.uint64),
        "leaves": np.empty((n, 2), np.uint64),
        "nodes": np.empty((max(2 * n - 1, 1), 10), np.uint64),
        "counters": np.empty(5, np.uint64),
        "root_aabb": np.empty(6, np.uint64),
    }
    root = np.zeros(1, np.uint64)
    secs = np.zeros(2)
    err = C.create_string_buffer(512)
    lib = _lib(which)
    if which == "restatement":
        fn = lib.oracle_lbvh_build
        args = [_p(pts), C.c_uint64(n), _p(out["source_index"]), _p(out["leaves"]), _p(out["nodes"]),
                _p(out["counters"]), _p(out["root_aabb"]), _p(root), err, C.c_uint64(512)]
    else:
        fn = lib.ref_lbvh_build
        args = [_p(pts), C.c_uint64(n), _p(out["source_index"]), _p(out["leaves"]), _p(out["nodes"]),
                _p(out["counters"]), _p(out["root_aabb"]), _p(root), _p(secs), err, C.c_uint64(512)]
    fn.restype = C.c_int
    rc = fn(*[a if not isinstance(a, int) else C.c_void_p(a) for a in args])
    if rc != 0:
        raise OracleError(rc, err.value.decode())
    out["root"] = int(root[0])
    out["seconds"] = secs
    if n == 0:
        out["nodes"] = out["nodes"][:0]
    return out


def ref_lbvh_certify(points: np.ndarray, snap) -> tuple[bool, str]:
    """The reference's own import_certified_snapshot on a device-built snapshot."""
    pts = np.ascontiguousarray(points, dtype=np.float64)
    n = pts.shape[0]
    err = C.create_string_buffer(512)
    fn = _lib("reference").ref_lbvh_certify
    fn.restype = C.c_int
    leaves = np.ascontiguousarray(snap.leaves, dtype=np.uint64)
    nodes = np.ascontiguousarray(snap.nodes, dtype=np.uint64)
    counters = np.ascontiguousarray(snap.counters, dtype=np.uint64)
    aabb = np.ascontiguousarray(snap.root_aabb, dtype=np.uint64)
    rc = fn(C.c_void_p(_p(pts)), C.c_uint64(n), C.c_void_p(_p(leaves)), C.c_void_p(_p(nodes)),
            C.c_void_p(_p(counters)), C.c_void_p(_p(aabb)), C.c_uint64(int(snap.root)), err, C.c_uint64(512))
    return rc == 0, err.value.decode()


def _text_call(fn_name: str, which: str, pts: np.ndarray, *extra) -> str:
    """Calls a text-blob oracle entry point, growing the buffer when needed."""
    lib = _lib(which)
    fn = getattr(lib, fn_name)
    fn.restype = C.c_int
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    cap = 1 << 20
    for _ in range(3):
        buf = C.create_string_buffer(cap)
        needed = C.c_uint64(0)
        err = C.create_string_buffer(512)
        secs = np.zeros(4)
        args = [C.c_void_p(_p(pts)), C.c_uint64(len(pts)), *[C.c_uint64(x) for x in extra], buf,
                C.c_uint64(cap), C.byref(needed)]
        if which == "reference":
            args.append(C.c_void_p(_p(secs)))
        args += [err, C.c_uint64(512)]
        rc = fn(*args)
        if rc != 0:
            raise OracleError(rc, err.value.decode())
        if needed.value == 0:
            _text_call.seconds = secs
            return buf.value.decode()
        cap = int(needed.value) + 16
    raise RuntimeError("oracle output did not fit")


def classify(points_canonical: np.ndarray, supports: np.ndarray) -> np.ndarray:
    """Exact classification of supports (rows: size, id0..id3; PointIds of the canonical
    cloud) against every point: rows (status 0 minimal / 1 not, strict interior count,
    complete shell count, least extra shell PointId or 0xffffffff, first 10 interior ids).
    `points_canonical` must already be in PointId order."""
    lib = _lib("restatement")
    fn = lib.oracle_classify
    fn.restype = C.c_int
    pts = np.ascontiguousarray(points_canonical, dtype=np.float64)
    sup = np.ascontiguousarray(supports, dtype=np.uint32)
    out = np.zeros((len(sup), 14), np.uint32)
    err = C.create_string_buffer(512)
    rc = fn(C.c_void_p(_p(pts)), C.c_uint64(len(pts)), C.c_void_p(_p(sup)), C.c_uint64(len(sup)),
            C.c_void_p(_p(out)), err, C.c_uint64(512))
    if rc != 0:
        raise OracleError(rc, err.value.decode())
    return out


def ref_pairs_budget(points: np.ndarray, K: int, work_units: int) -> dict:
    """The reference's own pair stream on the whole cloud under a work-unit budget
    (oracle/ref_driver.cpp ref_pairs_budget): time to the budget and how far it got."""
    lib = _lib("reference")
    fn = lib.ref_pairs_budget
    fn.restype = C.c_int
    pts = np.ascontiguousarray(points, dtype=np.float64)
    st = np.zeros(6, np.uint64)
    sec = np.zeros(2)
    err = C.create_string_buffer(512)
    rc = fn(C.c_void_p(_p(pts)), C.c_uint64(len(pts)), C.c_uint64(K), C.c_uint64(work_units), C.c_void_p(_p(st)),
            C.c_void_p(_p(sec)), err, C.c_uint64(512))
    if rc != 0:
        raise OracleError(rc, err.value.decode())
    return {"complete": int(st[0]) == 0, "work_units": int(st[1]), "resolved_pairs": int(st[2]),
            "total_pairs": int(st[3]), "events": int(st[4]), "diagnostics": int(st[5]),
            "lbvh_s": float(sec[0]), "stream_s": float(sec[1])}


def knn(points: np.ndarray, k: int, which: str = "restatement") -> list[tuple[list[int], list[int], Fraction]]:
    """Per PointId p: (strict ids in (d, id) order, shell ids, cutoff squared distance)."""
    name = "oracle_knn" if which == "restatement" else "ref_knn"
    out = []
    for line in _text_call(name, which, points, k).splitlines():
        strict, shell, cut = line.split("|")
        num, den = cut.split()
        out.append(([int(x) for x in strict.split()], [int(x) for x in shell.split()], Fraction(int(num), int(den))))
    return out


def emst_forest(points: np.ndarray, which: str = "restatement") -> dict:
    """EMST edges, Boruvka minima/accepted per round and the compact k=1 forest."""
    name = "oracle_emst_forest" if which == "restatement" else "ref_emst_forest"
    r = {"edges": [], "minima": [], "accepted": [], "levels": [], "nodes": [], "children": [], "batches": [],
         "root": None}
    for line in _text_call(name, which, points).splitlines():
        t = line.split()
        if not t:
            continue
        tag, f = t[0], t[1:]
        if tag == "E":
            r["edges"].append((int(f[0]), int(f[1]), Fraction(int(f[2]), int(f[3]))))
        elif tag == "M":
            r["minima"].append((int(f[0]), int(f[1]), int(f[2]), int(f[3]), int(f[4]), Fraction(int(f[5]), int(f[6]))))
        elif tag == "A":
            r["accepted"].append(tuple(int(x) for x in f))
        elif tag == "L":
            r["levels"].append(Fraction(int(f[0]), int(f[1])))
        elif tag == "N":
            r["nodes"].append(tuple(int(x) for x in f))
        elif tag == "C":
            r["children"] = [int(x) for x in f]
        elif tag == "B":
            r["batches"].append(tuple(int(x) for x in f))
        elif tag == "R":
            r["root"] = int(f[0])
    return r


def parse_pairs(txt: str) -> dict:
    """Pair-support records: events (u, v, closed_rank, exterior, level, center, interior)
    and diagnostics (u, v, shell, witness, min_rank, observed_rank, exterior, level, center, interior)."""
    events, diags, status = [], [], None
    for line in txt.splitlines():
        head, _, tail = line.partition("|")
        t = head.split()
        if not t:
            continue
        ids = tuple(int(x) for x in tail.split())
        if t[0] == "P":
            center = tuple(Fraction(int(t[7 + a]), int(t[10])) for a in range(3))
            events.append((int(t[1]), int(t[2]), int(t[3]), int(t[4]), Fraction(int(t[5]), int(t[6])), center, ids))
        elif t[0] == "D":
            center = tuple(Fraction(int(t[10 + a]), int(t[13])) for a in range(3))
            diags.append((*(int(x) for x in t[1:8]), Fraction(int(t[8]), int(t[9])), center, ids))
        elif t[0] == "S":
            status = t[1]
    return {"events": events, "diagnostics": diags, "status": status}


def pairs(points: np.ndarray, K: int = 10, which: str = "restatement") -> dict:
    name = "oracle_pairs" if which == "restatement" else "ref_pairs"
    return parse_pairs(_text_call(name, which, points, K))


def parse_higher(txt: str) -> dict:
    """Higher-support records: events (size, ids, closed_rank, exterior, level, center, interior)
    and diagnostics (size, ids, shell, witness, min_rank, observed_rank, exterior, level, center, interior)."""
    events, diags, status = [], [], None
    for line in txt.splitlines():
        head, _, tail = line.partition("|")
        t = head.split()
        if not t:
            continue
        ids = tuple(int(x) for x in tail.split())
        if t[0] in ("H", "G"):
            m = int(t[1])
            sup = tuple(int(x) for x in t[2:2 + m])
            r = t[2 + m:]
            if t[0] == "H":
                center = tuple(Fraction(int(r[4 + a]), int(r[7])) for a in range(3))
                events.append((m, sup, int(r[0]), int(r[1]), Fraction(int(r[2]), int(r[3])), center, ids))
            else:
                center = tuple(Fraction(int(r[7 + a]), int(r[10])) for a in range(3))
                diags.append((m, sup, *(int(x) for x in r[:5]), Fraction(int(r[5]), int(r[6])), center, ids))
        elif t[0] == "S":
            status = t[1]
    return {"events": events, "diagnostics": diags, "status": status}


def higher(points: np.ndarray, K: int = 10, which: str = "restatement") -> dict:
    name = "oracle_higher" if which == "restatement" else "ref_higher"
    return parse_higher(_text_call(name, which, points, K))


def hierarchy(pts: np.ndarray, K: int, which: str = "restatement") -> str:
    """The direct chain (facade, event journal, arm seeds, forest journal) as text:
    the restatement (oracle_hierarchy) or the reference's own code (ref_hierarchy)."""
    fn = "oracle_hierarchy" if which == "restatement" else "ref_hierarchy"
    return _text_call(fn, which, pts, K)
