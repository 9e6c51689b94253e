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

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT = os.path.join(HERE, "lib", "libehgp_oracle.so")
REFERENCE = os.path.join(HERE, "_ref", "libehgp_ref.so")

_libs: dict[str, C.CDLL] = {}


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
