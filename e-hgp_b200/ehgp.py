"""Host-side Python mirror of the C ABI in include/ehgp.h (ctypes).

This is how tests, the smoke check and bench.py drive the sm_100a library.
It mirrors the reference's GPU context interface for the product path
(Ludwig-H/E-HGP, morsehgp3d/include/morsehgp3d/gpu/morton_lbvh_build.hpp:185-208):
a context is created for a maximum point count and then builds clouds; a
failure raises, and a CUDA failure poisons the context.

Error mapping follows the reference's exceptions:
    EHGP_ERR_INVALID_ARGUMENT -> InvalidArgument (std::invalid_argument)
    EHGP_ERR_DUPLICATE_POINT  -> DuplicatePoint  (std::invalid_argument)
    EHGP_ERR_CAPACITY         -> CapacityError   (std::length_error)
    anything else             -> EhgpError

The library is loaded from e-hgp_b200/lib/libehgp_b200.so; there is no
fallback: if it is missing, `load()` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libehgp_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "ehgp.h")

STATUS = {
    0: "EHGP_OK", 1: "EHGP_ERR_INVALID_ARGUMENT", 2: "EHGP_ERR_DUPLICATE_POINT",
    3: "EHGP_ERR_CAPACITY", 4: "EHGP_ERR_OUT_OF_MEMORY", 5: "EHGP_ERR_TIMEOUT",
    6: "EHGP_ERR_DEGENERATE", 7: "EHGP_ERR_NUMERIC_RANGE", 8: "EHGP_ERR_CUDA",
    9: "EHGP_ERR_POISONED", 10: "EHGP_ERR_NOT_BUILT",
}


class EhgpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


class InvalidArgument(EhgpError, ValueError):
    pass


class DuplicatePoint(InvalidArgument):
    pass


class CapacityError(EhgpError):
    pass


class NumericRange(EhgpError):
    pass


class DegenerateError(EhgpError):
    """Relevant extra-shell diagnostics, or a strict-arm descent that cannot be certified."""


_ERRORS = {1: InvalidArgument, 2: DuplicatePoint, 3: CapacityError, 6: DegenerateError, 7: NumericRange}


class Limits(C.Structure):
    _fields_ = [("max_points", C.c_uint64), ("hbm_fraction", C.c_double)]


class LbvhOut(C.Structure):
    _fields_ = [
        ("source_index", C.c_void_p), ("leaves", C.c_void_p), ("nodes", C.c_void_p),
        ("counters", C.c_void_p), ("root_aabb_bits", C.c_void_p), ("root_node_index", C.c_void_p),
    ]


class KnnOut(C.Structure):
    _fields_ = [("ids", C.c_void_p), ("meta", C.c_void_p), ("cutoff_num", C.c_void_p)]


class EmstOut(C.Structure):
    _fields_ = [("u", C.c_void_p), ("v", C.c_void_p), ("squared_length_num", C.c_void_p),
                ("rounds", C.c_void_p), ("minima", C.c_void_p), ("minima_capacity", C.c_uint64),
                ("minima_count", C.c_void_p)]


class K1ForestOut(C.Structure):
    _fields_ = [("level_num", C.c_void_p), ("nodes", C.c_void_p), ("child_ids", C.c_void_p),
                ("batches", C.c_void_p), ("counts", C.c_void_p), ("root_node_id", C.c_void_p)]


class PairsOut(C.Structure):
    _fields_ = [("records", C.c_void_p), ("level_num", C.c_void_p), ("capacity", C.c_uint64),
                ("count", C.c_void_p)]


PAIR_RECORD = np.dtype([("u", "<u4"), ("v", "<u4"), ("interior_count", "<u4"), ("shell_count", "<u4"),
                        ("extra_shell_witness", "<u4"), ("interior_ids", "<u4", 9), ("reserved", "<u4", 2)])
assert PAIR_RECORD.itemsize == 64


class HigherOut(C.Structure):
    _fields_ = [("records", C.c_void_p), ("capacity", C.c_uint64), ("count", C.c_void_p)]


HIGHER_RECORD = np.dtype([("size", "<u4"), ("ids", "<u4", 4), ("interior_count", "<u4"), ("shell_count", "<u4"),
                          ("extra_shell_witness", "<u4"), ("interior_ids", "<u4", 8)])
assert HIGHER_RECORD.itemsize == 64


class HierCounts(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in ("events", "diagnostics", "journal_batches", "role_records", "families",
                                          "arm_seeds", "birth_records", "nodes", "children", "arm_bindings",
                                          "saddle_records", "atomic_groups", "final_roots")] + \
               [("decision", C.c_uint32), ("k_eff", C.c_uint32), ("vertical_assignments", C.c_uint64)]


def _u4(*names):
    return np.dtype([(nm, "<u4") for nm in names])


# Record layouts of include/ehgp.h (direct Morse hierarchy).
EVENT_RECORD = np.dtype([("support_size", "<u4"), ("support_ids", "<u4", 4), ("interior_count", "<u4"),
                         ("closed_rank", "<u4"), ("interior_ids", "<u4", 9)])
JOURNAL_BATCH = _u4("order", "level_event", "role_offset", "role_count", "birth_roles", "saddle_roles")
ROLE_RECORD = _u4("batch", "projection", "role")
FAMILY_RECORD = _u4("event", "projection", "role_record", "batch", "order", "arm_offset", "arm_count")
FOREST_NODE = _u4("order", "level_event", "kind", "child_offset", "child_count", "birth_record", "atomic_group")
FOREST_BIRTH = _u4("projection", "batch", "order", "handle", "order_one_node")
FOREST_BINDING = _u4("arm_seed", "family", "carrier", "prior_root")
FOREST_SADDLE = _u4("family", "event", "batch", "arm_offset", "arm_count", "carriers", "latent", "prior_roots",
                    "group")
FOREST_GROUP = _u4("batch", "saddle_offset", "saddle_count", "frozen", "latent", "prior_roots", "child_offset",
                   "child_count", "created_node", "result_node", "kind")
FOREST_BATCH = _u4("order", "level_event", "birth_offset", "birth_count", "saddle_offset", "saddle_count",
                   "group_offset", "group_count", "pre_carriers", "pre_roots", "post_carriers", "post_roots")
FOREST_ROOT = _u4("order", "handle", "node")
VERTICAL_ASSIGNMENT = _u4("source_node", "target_node", "source_order", "level_event")
ABSENT = 0xFFFFFFFF

_HIER_FIELDS = [("events", EVENT_RECORD, "events"), ("journal_batches", JOURNAL_BATCH, "journal_batches"),
                ("roles", ROLE_RECORD, "role_records"), ("families", FAMILY_RECORD, "families"),
                ("arm_removed", np.dtype("<u4"), "arm_seeds"), ("nodes", FOREST_NODE, "nodes"),
                ("children", np.dtype("<u4"), "children"), ("births", FOREST_BIRTH, "birth_records"),
                ("bindings", FOREST_BINDING, "arm_bindings"), ("saddles", FOREST_SADDLE, "saddle_records"),
                ("groups", FOREST_GROUP, "atomic_groups"), ("batches", FOREST_BATCH, "journal_batches"),
                ("roots", FOREST_ROOT, "final_roots"),
                ("vertical", VERTICAL_ASSIGNMENT, "vertical_assignments")]


class HierOut(C.Structure):
    _fields_ = [(name, C.c_void_p) for name, _, _ in _HIER_FIELDS]


class ServerLimits(C.Structure):
    _fields_ = [("workers", C.c_uint32), ("max_points", C.c_uint64), ("hbm_fraction", C.c_double)]


class CloudDesc(C.Structure):
    _fields_ = [("xyz", C.c_void_p), ("n", C.c_uint64), ("dtype", C.c_uint32), ("K", C.c_uint32)]


class RequestStats(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("points", C.c_uint64), ("K", C.c_uint32),
                ("worker", C.c_uint32), ("queued_ms", C.c_double), ("service_ms", C.c_double),
                ("latency_ms", C.c_double), ("device_ms", C.c_double), ("counts", HierCounts)]


class ServedOut(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("nodes", "children", "batches", "roots", "vertical", "node_supports",
                                          "emst_u", "emst_v")]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


def limbs_to_int(a: np.ndarray) -> int:
    """Little-endian 64-bit limbs -> Python int."""
    v = 0
    for w in reversed([int(x) for x in a]):
        v = (v << 64) | w
    return v


_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads the sm_100a library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run `python e-hgp_b200/build.py`")
    lib = C.CDLL(path)
    P = C.c_void_p
    sigs = {
        "ehgp_ctx_create": (C.c_int, [C.c_int, C.POINTER(Limits), C.POINTER(P)]),
        "ehgp_ctx_destroy": (C.c_int, [P]),
        "ehgp_last_error": (C.c_char_p, [P]),
        "ehgp_status_string": (C.c_char_p, [C.c_int]),
        "ehgp_ctx_device_bytes": (C.c_uint64, [P]),
        "ehgp_lbvh_build": (C.c_int, [P, P, C.c_uint64, C.POINTER(LbvhOut)]),
        "ehgp_lbvh_build_f32": (C.c_int, [P, P, C.c_uint64, C.POINTER(LbvhOut)]),
        "ehgp_lbvh_build_device": (C.c_int, [P, P, C.c_uint64, C.POINTER(LbvhOut)]),
        "ehgp_last_timing": (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
        "ehgp_cloud_scale": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "ehgp_knn": (C.c_int, [P, C.c_uint32, C.POINTER(KnnOut)]),
        "ehgp_emst": (C.c_int, [P, C.POINTER(EmstOut)]),
        "ehgp_k1_forest": (C.c_int, [P, C.POINTER(K1ForestOut)]),
        "ehgp_pairs": (C.c_int, [P, C.c_uint32, C.POINTER(PairsOut)]),
        "ehgp_higher": (C.c_int, [P, C.c_uint32, C.POINTER(HigherOut)]),
        "ehgp_higher_stats": (C.c_int, [P, C.POINTER(C.c_double), P, C.c_uint32]),
        "ehgp_step_begin": (C.c_int, [P]),
        "ehgp_step_end": (C.c_int, [P, C.POINTER(C.c_double)]),
        "ehgp_kernel_stats": (C.c_int, [P, C.POINTER(C.c_double), P, C.c_uint32]),
        "ehgp_lbvh_build_noalloc": (C.c_int, [P, C.c_uint64, C.POINTER(LbvhOut), P]),
        "ehgp_lbvh_noalloc_max_points": (C.c_uint64, []),
        "ehgp_lbvh_noalloc_scratch_bytes": (C.c_uint64, []),
        "ehgp_hierarchy": (C.c_int, [P, C.c_uint32, C.POINTER(HierCounts)]),
        "ehgp_hier_copy": (C.c_int, [P, C.POINTER(HierOut)]),
        "ehgp_event_level": (C.c_int, [P, C.c_uint64, P, P, C.POINTER(C.c_int32)]),
        "ehgp_hier_stats": (C.c_int, [P, P, P]),
        "ehgp_hier_schedule": (C.c_int, [P, C.c_uint32, C.c_uint32, C.c_uint32]),
        "ehgp_ctx_reserve": (C.c_int, [P, C.c_uint32, C.c_uint64]),
        "ehgp_ctx_regrowths": (C.c_uint64, [P]),
        "ehgp_tune": (C.c_int, [P, C.c_uint32, C.c_uint64]),
        "ehgp_event_supports": (C.c_int, [P, P, C.c_uint64, P]),
        "ehgp_predicate_eval": (C.c_int, [P, C.c_uint32, P, C.c_uint32, P]),
        "ehgp_ctx_counters": (C.c_int, [P, P, C.c_uint32]),
        "ehgp_checkpoint_save": (C.c_int, [P, C.c_uint32, C.c_char_p]),
        "ehgp_checkpoint_load": (C.c_int, [P, C.c_char_p, C.POINTER(C.c_uint32)]),
        "ehgp_server_create": (C.c_int, [C.c_int, C.POINTER(ServerLimits), C.POINTER(P)]),
        "ehgp_server_destroy": (C.c_int, [P]),
        "ehgp_cloud_submit": (C.c_int, [P, C.POINTER(CloudDesc), C.POINTER(C.c_uint64)]),
        "ehgp_poll": (C.c_int, [P, C.c_uint64, C.POINTER(C.c_int32)]),
        "ehgp_wait": (C.c_int, [P, C.c_uint64, C.c_uint64, C.POINTER(C.c_int32)]),
        "ehgp_request_info": (C.c_int, [P, C.c_uint64, C.POINTER(RequestStats)]),
        "ehgp_request_error": (C.c_char_p, [P, C.c_uint64]),
        "ehgp_result_copy": (C.c_int, [P, C.c_uint64, C.POINTER(ServedOut)]),
        "ehgp_result_release": (C.c_int, [P, C.c_uint64]),
        "ehgp_server_info": (C.c_int, [P, P, C.c_uint32]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols(header: str = HEADER) -> list[str]:
    """Names of the functions include/ehgp.h declares."""
    import re
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ehgp_[a-z0-9_]+)\s*\(", text)))


@dataclass
class LbvhSnapshot:
    """Reference-layout MortonLbvhSnapshot (include/morsehgp3d/spatial/lbvh.hpp:109-121)."""
    source_index: np.ndarray   # (n,) u64: input index of PointId p
    leaves: np.ndarray         # (n, 2) u64: (Morton code, PointId)
    nodes: np.ndarray          # (2n-1, 10) u64: lower[3], upper[3], left, right, begin, end
    counters: np.ndarray       # (5,) u64
    root_aabb: np.ndarray      # (6,) u64 binary64 words
    root: int


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _empty_snapshot(n: int) -> tuple[LbvhSnapshot, np.ndarray, LbvhOut]:
    snap = LbvhSnapshot(
        np.empty(n, np.uint64), np.empty((n, 2), np.uint64),
        np.empty((max(2 * n - 1, 0), 10), np.uint64), np.empty(5, np.uint64),
        np.empty(6, np.uint64), 0)
    root = np.zeros(1, np.uint64)
    out = LbvhOut(_ptr(snap.source_index), _ptr(snap.leaves), _ptr(snap.nodes),
                  _ptr(snap.counters), _ptr(snap.root_aabb), _ptr(root))
    return snap, root, out


def lbvh_build_noalloc(points: np.ndarray, stream: int = 0) -> LbvhSnapshot:
    """ehgp_lbvh_build_noalloc: the LBVH build without any allocation by the
    library, for callers that may not call cudaMalloc.  At most
    ehgp_lbvh_noalloc_max_points() points; runs on the current device."""
    lib = load()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    if pts.ndim != 2 or pts.shape[1] != 3:
        raise InvalidArgument(1, "points must have shape (n, 3)")
    snap, root, out = _empty_snapshot(pts.shape[0])
    st = lib.ehgp_lbvh_build_noalloc(_ptr(pts), pts.shape[0], C.byref(out), C.c_void_p(stream))
    if st != 0:
        raise _ERRORS.get(st, EhgpError)(st, "ehgp_lbvh_build_noalloc failed")
    snap.root = int(root[0])
    return snap


class Context:
    """One device context (mirrors gpu::MortonLbvhBuildContext)."""

    def __init__(self, max_points: int, device: int = 0, hbm_fraction: float = 0.8):
        self.lib = load()
        self._h = C.c_void_p()
        lim = Limits(max_points, hbm_fraction)
        st = self.lib.ehgp_ctx_create(device, C.byref(lim), C.byref(self._h))
        if st != 0:
            raise _ERRORS.get(st, EhgpError)(st, "context creation failed")
        self.max_points = max_points
        self.device = device

    def close(self) -> None:
        if self._h:
            self.lib.ehgp_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != 0:
            msg = self.lib.ehgp_last_error(self._h).decode()
            raise _ERRORS.get(st, EhgpError)(st, msg)

    @property
    def device_bytes(self) -> int:
        return int(self.lib.ehgp_ctx_device_bytes(self._h))

    def reserve(self, stage: int, records: int) -> None:
        """ehgp_ctx_reserve: record capacity of the pair (0) or triple/quad (1) buffers."""
        self._check(self.lib.ehgp_ctx_reserve(self._h, stage, records))

    TUNE_HIGHER_LIST = 1

    def tune(self, knob: int, value: int) -> None:
        """ehgp_tune: a tuning knob of later calls (results never depend on it)."""
        self._check(self.lib.ehgp_tune(self._h, knob, value))

    def counters(self) -> dict:
        """ehgp_ctx_counters: device bytes, regrowths, pair and triple/quad enumerations run."""
        v = np.zeros(4, np.uint64)
        self._check(self.lib.ehgp_ctx_counters(self._h, _ptr(v), 4))
        return dict(zip(("device_bytes", "regrowths", "pair_runs", "higher_runs"), (int(x) for x in v)))

    def checkpoint_save(self, path: str, K: int = 10) -> None:
        """ehgp_checkpoint_save: cloud, K and support records of the resident cloud to `path`."""
        self._check(self.lib.ehgp_checkpoint_save(self._h, K, os.fsencode(path)))

    def checkpoint_load(self, path: str) -> int:
        """ehgp_checkpoint_load: the cloud and support records of a checkpoint; returns its K."""
        K = C.c_uint32()
        self._check(self.lib.ehgp_checkpoint_load(self._h, os.fsencode(path), C.byref(K)))
        with open(path, "rb") as f:  # header: magic, version, K, point count
            self.n = int(np.frombuffer(f.read(24)[16:24], np.uint64)[0])
        return K.value

    def regrowths(self) -> int:
        """Second enumeration passes after a record buffer grew (count -> allocate -> emit)."""
        return int(self.lib.ehgp_ctx_regrowths(self._h))

    def step_begin(self) -> None:
        self._check(self.lib.ehgp_step_begin(self._h))

    def step_end(self) -> float:
        ms = C.c_double()
        self._check(self.lib.ehgp_step_end(self._h, C.byref(ms)))
        return ms.value

    def kernel_stats(self) -> tuple[float, np.ndarray]:
        ms = C.c_double()
        st = np.zeros(8, np.uint64)
        self._check(self.lib.ehgp_kernel_stats(self._h, C.byref(ms), _ptr(st), 8))
        return ms.value, st

    def last_timing(self) -> tuple[float, int]:
        ms, launches = C.c_double(), C.c_uint64()
        self._check(self.lib.ehgp_last_timing(self._h, C.byref(ms), C.byref(launches)))
        return ms.value, launches.value

    def lbvh_build(self, points: np.ndarray, outputs: bool = True) -> LbvhSnapshot | None:
        """Canonical cloud + exact Morton LBVH (ehgp_lbvh_build / _f32).

        points: (n, 3) float64 or float32 array.  With outputs=False only the
        device-resident index is built (nothing is copied back)."""
        pts = np.ascontiguousarray(points)
        if pts.ndim != 2 or pts.shape[1] != 3:
            raise InvalidArgument(1, "points must have shape (n, 3)")
        n = pts.shape[0]
        if outputs:
            snap = LbvhSnapshot(
                np.empty(n, np.uint64), np.empty((n, 2), np.uint64),
                np.empty((max(2 * n - 1, 0), 10), np.uint64), np.empty(5, np.uint64),
                np.empty(6, np.uint64), 0)
            root = np.zeros(1, np.uint64)
            out = LbvhOut(_ptr(snap.source_index), _ptr(snap.leaves), _ptr(snap.nodes),
                          _ptr(snap.counters), _ptr(snap.root_aabb), _ptr(root))
        else:
            snap, out = None, LbvhOut(None, None, None, None, None, None)
        if pts.dtype == np.float32:
            st = self.lib.ehgp_lbvh_build_f32(self._h, _ptr(pts), n, C.byref(out))
        else:
            pts = pts.astype(np.float64, copy=False)
            st = self.lib.ehgp_lbvh_build(self._h, _ptr(pts), n, C.byref(out))
        self._check(st)
        self.n = n
        if snap is not None:
            snap.root = int(root[0])
        return snap

    def lbvh_build_dlpack(self, points, outputs: bool = False) -> LbvhSnapshot | None:
        """Zero-copy device input (ehgp_lbvh_build_device): `points` is a DLPack producer or a
        __cuda_array_interface__ object (a torch or CuPy CUDA array) of shape (n, 3) on this
        context's device.  binary64 points are read in place; binary32 points are widened
        exactly on the device first (one temporary).  Work pending on torch's current stream
        (the producer's) is waited for before the library's stream reads the points."""
        import torch
        if isinstance(points, torch.Tensor):
            t = points
        elif hasattr(points, "__dlpack__") or type(points).__name__ == "PyCapsule":
            t = torch.from_dlpack(points)  # a producer, or a raw DLPack capsule
        elif hasattr(points, "__cuda_array_interface__"):
            t = torch.as_tensor(points, device=f"cuda:{self.device}")
        else:
            raise InvalidArgument(1, "points must be a CUDA array (DLPack or __cuda_array_interface__)")
        if not t.is_cuda or t.device.index != self.device:
            raise InvalidArgument(1, f"points must be on cuda:{self.device}")
        if t.ndim != 2 or t.shape[1] != 3:
            raise InvalidArgument(1, "points must have shape (n, 3)")
        if t.dtype == torch.float32:
            t = t.to(torch.float64)
        elif t.dtype != torch.float64:
            raise InvalidArgument(1, "points must be binary32 or binary64")
        t = t.contiguous()
        torch.cuda.current_stream(t.device).synchronize()
        n = int(t.shape[0])
        if outputs:
            snap = LbvhSnapshot(
                np.empty(n, np.uint64), np.empty((n, 2), np.uint64),
                np.empty((max(2 * n - 1, 0), 10), np.uint64), np.empty(5, np.uint64),
                np.empty(6, np.uint64), 0)
            root = np.zeros(1, np.uint64)
            out = LbvhOut(_ptr(snap.source_index), _ptr(snap.leaves), _ptr(snap.nodes),
                          _ptr(snap.counters), _ptr(snap.root_aabb), _ptr(root))
        else:
            snap, out = None, LbvhOut(None, None, None, None, None, None)
        self._check(self.lib.ehgp_lbvh_build_device(self._h, C.c_void_p(t.data_ptr()), n, C.byref(out)))
        self.n = n
        if snap is not None:
            snap.root = int(root[0])
        return snap

    # ---- exact geometry of the resident cloud ----------------------------------
    def scale(self) -> tuple[int, bool]:
        s, valid = C.c_int32(), C.c_int32()
        self._check(self.lib.ehgp_cloud_scale(self._h, C.byref(s), C.byref(valid)))
        return s.value, bool(valid.value)

    def knn(self, k: int) -> dict:
        """ehgp_knn: per PointId, canonical top-k ids, (strict, shell) counts and
        the exact cutoff as a Fraction."""
        from fractions import Fraction
        n = self.n
        ids = np.empty((n, k), np.uint32)
        meta = np.empty((n, 2), np.uint32)
        cut = np.empty((n, 4), np.uint64)
        out = KnnOut(_ptr(ids), _ptr(meta), _ptr(cut))
        self._check(self.lib.ehgp_knn(self._h, k, C.byref(out)))
        S, _ = self.scale()
        den = 1 << (2 * S)
        return {"ids": ids, "meta": meta, "cutoff_num": cut,
                "cutoff": [Fraction(limbs_to_int(c), den) for c in cut]}

    def emst(self, with_minima: bool = True) -> dict:
        """ehgp_emst: EMST edges in (squared length, u, v) order with exact lengths."""
        n = self.n
        m = max(n - 1, 0)
        u = np.empty(max(m, 1), np.uint32)
        v = np.empty(max(m, 1), np.uint32)
        D = np.empty((max(m, 1), 4), np.uint64)
        rounds = np.zeros(1, np.uint32)
        cap = 2 * n if with_minima else 0
        minima = np.empty((max(cap, 1), 4), np.uint32)
        mcount = np.zeros(1, np.uint64)
        out = EmstOut(_ptr(u), _ptr(v), _ptr(D), _ptr(rounds), _ptr(minima) if cap else None, cap, _ptr(mcount))
        self._check(self.lib.ehgp_emst(self._h, C.byref(out)))
        mc = int(mcount[0]) if cap else 0
        return {"u": u[:m], "v": v[:m], "D": D[:m], "rounds": int(rounds[0]), "minima": minima[:mc]}

    def pairs(self, K: int = 10) -> dict:
        """ehgp_pairs: relevant pair supports in (u, v) order (reference-layout records)."""
        cnt = np.zeros(1, np.uint64)
        self._check(self.lib.ehgp_pairs(self._h, K, C.byref(PairsOut(None, None, 0, _ptr(cnt)))))
        m = int(cnt[0])
        recs = np.zeros(max(m, 1), PAIR_RECORD)
        lv = np.zeros((max(m, 1), 4), np.uint64)
        self._check(self.lib.ehgp_pairs(self._h, K, C.byref(PairsOut(_ptr(recs), _ptr(lv), m, _ptr(cnt)))))
        return {"records": recs[:m], "level_num": lv[:m]}

    def higher(self, K: int = 10) -> np.ndarray:
        """ehgp_higher: relevant minimal triple/quad supports in (size, ids) order."""
        cnt = np.zeros(1, np.uint64)
        self._check(self.lib.ehgp_higher(self._h, K, C.byref(HigherOut(None, 0, _ptr(cnt)))))
        m = int(cnt[0])
        recs = np.zeros(max(m, 1), HIGHER_RECORD)
        self._check(self.lib.ehgp_higher(self._h, K, C.byref(HigherOut(_ptr(recs), m, _ptr(cnt)))))
        return recs[:m]

    def higher_stats(self) -> tuple[float, np.ndarray]:
        """Kernel time (ms) of the last triple/quad enumeration and its 14 work counters
        (include/ehgp.h, ehgp_higher_stats)."""
        ms = C.c_double()
        st = np.zeros(14, np.uint64)
        self._check(self.lib.ehgp_higher_stats(self._h, C.byref(ms), _ptr(st), 14))
        return ms.value, st

    def hierarchy(self, K: int = 10, arrays: bool = True) -> dict:
        """ehgp_hierarchy: facade, event journal, arm seeds and forest journal on the resident cloud.

        Raises DegenerateError (EHGP_ERR_DEGENERATE) when relevant extra-shell
        diagnostics stop the chain; `last_hier_counts` then holds the facade counts."""
        cnt = HierCounts()
        st = self.lib.ehgp_hierarchy(self._h, K, C.byref(cnt))
        self.last_hier_counts = {f: getattr(cnt, f) for f, _ in HierCounts._fields_}
        self._check(st)
        out = dict(self.last_hier_counts)
        if arrays:
            bufs = {}
            cnts = self.last_hier_counts
            for name, dt, cf in _HIER_FIELDS:
                bufs[name] = np.zeros(max(int(cnts[cf]), 1), dt)
            ho = HierOut(*[_ptr(bufs[name]) for name, _, _ in _HIER_FIELDS])
            self._check(self.lib.ehgp_hier_copy(self._h, C.byref(ho)))
            for name, _, cf in _HIER_FIELDS:
                out[name] = bufs[name][:int(cnts[cf])]
        return out

    def hier_schedule(self, chunk_batches: int = 0, part_arms: int = 0, host_threads: int = 0) -> None:
        """ehgp_hier_schedule: chunk, descent-part and thread counts of later hierarchy calls
        (0 = default); the result never depends on them."""
        self._check(self.lib.ehgp_hier_schedule(self._h, chunk_batches, part_arms, host_threads))

    def hier_stats(self) -> dict:
        """Timing and work counters of the last hierarchy call."""
        ms = np.zeros(25)
        st = np.zeros(15, np.uint64)
        self._check(self.lib.ehgp_hier_stats(self._h, _ptr(ms), _ptr(st)))
        return {"device_ms": ms[0], "descent_ms": ms[1], "forest_ms": ms[2], "slowest_order_ms": ms[3],
                "facade_ties_ms": ms[4], "host_orders_ms": ms[5], "host_offsets_ms": ms[6], "host_vertical_ms": ms[7],
                "order_ms": [float(x) for x in ms[8:24] if x > 0], "step_kernels_ms": float(ms[24]),
                "step_node_visits": int(st[13]), "step_launches": int(st[14]),
                "arms": int(st[0]),
                "descent_steps": int(st[1]), "exact_boundaries": int(st[2]), "events": int(st[3]),
                "first_misses": int(st[4]), "descent_rounds": int(st[5]),
                "slow": {k: int(v) for k, v in zip(("exhaustive_miniball", "exact_hull", "exact_side", "exact_level",
                                                    "exact_band", "exact_cutoff", "equal_cutoff"), st[6:13])}}

    def event_level(self, event: int):
        """Exact level of a facade event as a Fraction (cloud units)."""
        from fractions import Fraction
        num = np.zeros(36, np.uint64)
        den = np.zeros(36, np.uint64)
        S = C.c_int32()
        self._check(self.lib.ehgp_event_level(self._h, event, _ptr(num), _ptr(den), C.byref(S)))
        def signed(a):
            v = limbs_to_int(a)
            return v - (1 << (64 * 36)) if v >> (64 * 36 - 1) else v
        return Fraction(signed(num), signed(den) << (2 * S.value))

    PRED_SUPPORT_SIDE, PRED_SUPPORT_STATUS, PRED_LEVEL_CMP, PRED_DISTANCE_CMP = 1, 2, 3, 4

    def predicate(self, kind: int, ids) -> tuple[int, bool]:
        """ehgp_predicate_eval: (result, decided by the FP64 filter)."""
        a = np.ascontiguousarray(ids, dtype=np.uint32)
        out = np.zeros(2, np.int32)
        self._check(self.lib.ehgp_predicate_eval(self._h, kind, _ptr(a), len(a), _ptr(out)))
        return int(out[0]), bool(out[1])

    def event_supports(self, events: np.ndarray) -> np.ndarray:
        """ehgp_event_supports: (size, ids[4]) of facade events of the last hierarchy."""
        ev = np.ascontiguousarray(events, dtype=np.uint32)
        out = np.zeros((max(len(ev), 1), 5), np.uint32)
        self._check(self.lib.ehgp_event_supports(self._h, _ptr(ev), len(ev), _ptr(out)))
        return out[:len(ev)]

    def served_result(self, K: int = 10) -> dict:
        """The payload a served request carries, computed on this context for the
        resident cloud (EMST, hierarchy arrays, node level supports)."""
        n = self.n
        u = np.zeros(max(n - 1, 1), np.uint32)
        v = np.zeros(max(n - 1, 1), np.uint32)
        self._check(self.lib.ehgp_emst(self._h, C.byref(EmstOut(_ptr(u), _ptr(v), None, None, None, 0, None))))
        r = self.hierarchy(K, arrays=False)
        sizes = {"nodes": r["nodes"], "children": r["children"], "batches": r["journal_batches"],
                 "roots": r["final_roots"], "vertical": r["vertical_assignments"]}
        arr = {"nodes": np.zeros(max(sizes["nodes"], 1), FOREST_NODE),
               "children": np.zeros(max(sizes["children"], 1), np.uint32),
               "batches": np.zeros(max(sizes["batches"], 1), FOREST_BATCH),
               "roots": np.zeros(max(sizes["roots"], 1), FOREST_ROOT),
               "vertical": np.zeros(max(sizes["vertical"], 1), VERTICAL_ASSIGNMENT)}
        ho = HierOut(*[_ptr(arr[name]) if name in arr else None for name, _, _ in _HIER_FIELDS])
        self._check(self.lib.ehgp_hier_copy(self._h, C.byref(ho)))
        out = {k: a[:sizes[k]] for k, a in arr.items()}
        out["node_supports"] = self.event_supports(out["nodes"]["level_event"])
        out["emst_u"], out["emst_v"] = u[:n - 1], v[:n - 1]
        return out

    def k1_forest(self) -> dict:
        """ehgp_k1_forest on the last EMST: reference-layout compact forest arenas."""
        n = self.n
        m = max(n - 1, 1)
        lv = np.empty((m, 4), np.uint64)
        nodes = np.empty((m, 6), np.uint64)
        child = np.empty(2 * m, np.uint64)
        batches = np.empty((m, 7), np.uint64)
        counts = np.zeros(4, np.uint64)
        root = np.zeros(1, np.uint64)
        out = K1ForestOut(_ptr(lv), _ptr(nodes), _ptr(child), _ptr(batches), _ptr(counts), _ptr(root))
        self._check(self.lib.ehgp_k1_forest(self._h, C.byref(out)))
        L, N, Ch, B = (int(x) for x in counts)
        return {"level_num": lv[:L], "nodes": nodes[:N], "children": child[:Ch], "batches": batches[:B],
                "root": int(root[0])}


class Server:
    """Serving engine (include/ehgp.h ehgp_server_*): clouds are submitted asynchronously and
    run `workers` at a time on contexts of their own, admitted by device memory."""

    def __init__(self, workers: int = 4, max_points: int = 100_000, device: int = 0, hbm_fraction: float = 0.8):
        self.lib = load()
        h = C.c_void_p()
        lim = ServerLimits(workers, max_points, hbm_fraction)
        st = self.lib.ehgp_server_create(device, C.byref(lim), C.byref(h))
        if st != 0:
            raise _ERRORS.get(st, EhgpError)(st, "ehgp_server_create failed")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.ehgp_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, points: np.ndarray, K: int = 10) -> int:
        pts = np.ascontiguousarray(points)
        dtype = 1 if pts.dtype == np.float32 else 0
        if dtype == 0:
            pts = np.ascontiguousarray(pts, dtype=np.float64)
        rid = C.c_uint64()
        st = self.lib.ehgp_cloud_submit(self._h, C.byref(CloudDesc(pts.ctypes.data, len(pts), dtype, K)),
                                        C.byref(rid))
        if st != 0:
            raise _ERRORS.get(st, EhgpError)(st, "ehgp_cloud_submit refused the cloud")
        return rid.value

    def poll(self, rid: int) -> int:
        state = C.c_int32()
        st = self.lib.ehgp_poll(self._h, rid, C.byref(state))
        if st != 0:
            raise _ERRORS.get(st, EhgpError)(st, "ehgp_poll")
        return state.value

    def wait(self, rid: int, timeout_s: float = 600.0) -> int:
        """Waits for a request; returns its status (0 = complete)."""
        status = C.c_int32()
        st = self.lib.ehgp_wait(self._h, rid, int(timeout_s * 1e9), C.byref(status))
        if st != 0:
            raise _ERRORS.get(st, EhgpError)(st, "ehgp_wait")
        return status.value

    def info(self, rid: int) -> dict:
        s = RequestStats()
        st = self.lib.ehgp_request_info(self._h, rid, C.byref(s))
        if st != 0:
            raise _ERRORS.get(st, EhgpError)(st, "ehgp_request_info")
        out = {f: getattr(s, f) for f, _ in RequestStats._fields_ if f != "counts"}
        out["counts"] = {f: getattr(s.counts, f) for f, _ in HierCounts._fields_}
        out["error"] = self.lib.ehgp_request_error(self._h, rid).decode()
        return out

    def result(self, rid: int) -> dict:
        """Host copy of a completed request's result arrays."""
        inf = self.info(rid)
        if inf["state"] != REQ_DONE:
            raise _ERRORS.get(inf["status"], EhgpError)(inf["status"], inf["error"] or "request not complete")
        c = inf["counts"]
        n = int(inf["points"])
        res = {"nodes": np.zeros(max(c["nodes"], 1), FOREST_NODE), "children": np.zeros(max(c["children"], 1), "<u4"),
               "batches": np.zeros(max(c["journal_batches"], 1), FOREST_BATCH),
               "roots": np.zeros(max(c["final_roots"], 1), FOREST_ROOT),
               "vertical": np.zeros(max(c["vertical_assignments"], 1), VERTICAL_ASSIGNMENT),
               "node_supports": np.zeros((max(c["nodes"], 1), 5), "<u4"),
               "emst_u": np.zeros(max(n - 1, 1), "<u4"), "emst_v": np.zeros(max(n - 1, 1), "<u4")}
        out = ServedOut(*[_ptr(res[k]) for k, _ in ServedOut._fields_])
        st = self.lib.ehgp_result_copy(self._h, rid, C.byref(out))
        if st != 0:
            raise _ERRORS.get(st, EhgpError)(st, "ehgp_result_copy")
        sizes = {"nodes": c["nodes"], "children": c["children"], "batches": c["journal_batches"],
                 "roots": c["final_roots"], "vertical": c["vertical_assignments"], "node_supports": c["nodes"],
                 "emst_u": n - 1, "emst_v": n - 1}
        return {k: v[:sizes[k]] for k, v in res.items()}

    def release(self, rid: int) -> None:
        self.lib.ehgp_result_release(self._h, rid)

    def stats(self) -> dict:
        v = np.zeros(8, np.uint64)
        self.lib.ehgp_server_info(self._h, _ptr(v), 8)
        return dict(zip(("budget", "reserved", "held", "bytes_per_point", "queued", "running", "completed",
                         "memory_waits"), (int(x) for x in v)))


def _is_device_array(points) -> bool:
    if isinstance(points, np.ndarray):
        return False
    try:
        import torch
        if isinstance(points, torch.Tensor):
            return points.is_cuda
    except ImportError:
        pass
    return (hasattr(points, "__cuda_array_interface__") or hasattr(points, "__dlpack__")
            or type(points).__name__ == "PyCapsule")


def fit(points, K: int = 10, device: int = 0) -> dict:
    """One call from points to the hgp_reduced hierarchy, mirroring the front end the
    reference plans (morsehgp3d/docs/GPU_G4_ARCHITECTURE.md:269-294, `fit`): a host array, or a
    CUDA array by DLPack / __cuda_array_interface__ (read in place).  Returns the EMST edges, the
    forest nodes of orders 1..K with the supports of their levels, the child arena, forest
    batches, final roots, vertical maps, the hierarchy counts and the canonical points (PointId
    order, binary64) that the supports index."""
    if _is_device_array(points):
        import torch
        t = points if isinstance(points, torch.Tensor) else torch.from_dlpack(points)
        n = int(t.shape[0])
    else:
        points = np.ascontiguousarray(points)
        n = int(points.shape[0])
    with Context(max_points=max(n, 1), device=device) as ctx:
        snap = ctx.lbvh_build_dlpack(points, outputs=True) if _is_device_array(points) else ctx.lbvh_build(points)
        res = ctx.served_result(K)
        res["counts"] = dict(ctx.last_hier_counts)
        if _is_device_array(points):
            import torch
            t = points if isinstance(points, torch.Tensor) else torch.from_dlpack(points)
            host = t.detach().to("cpu", torch.float64).numpy()
        else:
            host = np.asarray(points, dtype=np.float64)
        res["points"] = host[snap.source_index.astype(np.int64)]
        res["K"] = K
        return HierarchyResult(res)


class HierarchyResult(dict):
    """Result of `fit` (a dict of arrays) with on-demand cuts."""

    def node_levels(self, order: int):
        """Exact squared levels (Fractions) of the nodes of one order, by node index."""
        from fractions import Fraction
        P = self["points"]
        nodes = self["nodes"]
        sup = self["node_supports"]
        out = {}
        for i in np.nonzero(nodes["order"] == order)[0]:
            m = int(sup[i, 0])
            if m == 0:
                out[int(i)] = Fraction(0)
                continue
            pts = [[Fraction(float(x)) for x in P[int(j)]] for j in sup[i, 1:1 + m]]
            out[int(i)] = _circumradius2(pts)
        return out

    def cut(self, order: int, level, closed: bool = True) -> list[int]:
        """Components of the order-`order` merge forest at squared level `level` (a number
        or Fraction): the nodes born at or below the level (strictly below when closed is
        False) whose parent, if any, is born above it; sorted node indices.  The cut of the
        reference's filtration (reference/morsehgp3d_oracle/gamma.py:213, GammaFiltration.cut;
        planned as result.cut(k, a), docs/GPU_G4_ARCHITECTURE.md:288-289), on the reduced forest."""
        from fractions import Fraction
        a = Fraction(level)
        lev = self.node_levels(order)
        nodes, ch = self["nodes"], self["children"]
        parent = {}
        for i in lev:
            if nodes["kind"][i] == 2:
                for c in ch[nodes["child_offset"][i]:nodes["child_offset"][i] + nodes["child_count"][i]]:
                    parent[int(c)] = i
        inside = (lambda x: x <= a) if closed else (lambda x: x < a)
        return sorted(i for i, x in lev.items() if inside(x) and (i not in parent or not inside(lev[parent[i]])))


def _circumradius2(pts):
    """Exact squared circumradius of 2-4 points (Fractions); a triangle's circle is centred in
    its plane."""
    a = pts[0]
    e = [[p[k] - a[k] for k in range(3)] for p in pts[1:]]
    dot = lambda u, v: sum(x * y for x, y in zip(u, v))
    if len(pts) == 2:
        return dot(e[0], e[0]) / 4
    cross = lambda u, v: [u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]]
    if len(pts) == 3:
        G11, G12, G22 = dot(e[0], e[0]), dot(e[0], e[1]), dot(e[1], e[1])
        A = G11 * G22 - G12 * G12
        N = [G22 * (G11 - G12) * e[0][k] + G11 * (G22 - G12) * e[1][k] for k in range(3)]
    else:
        c23, c31, c12 = cross(e[1], e[2]), cross(e[2], e[0]), cross(e[0], e[1])
        A = dot(e[0], c23)
        N = [dot(e[0], e[0]) * c23[k] + dot(e[1], e[1]) * c31[k] + dot(e[2], e[2]) * c12[k] for k in range(3)]
    return dot(N, N) / (4 * A * A)
