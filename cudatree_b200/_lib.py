"""ctypes binding of libcudatree_b200.so (C ABI in include/cudatree_b200.h).

The library is loaded from this package directory.  There is no CPU
fallback: if the library is missing or cannot be loaded, every entry point
raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcudatree_b200.so"

CT_OK = 0
CT_FIT_PLAIN = 0
CT_FIT_BATCHED = 1
CT_FIT_PROFILE = 1     # ct_fit_options.flags
CT_FIT_HOST_LOOP = 2
CT_FIT_NO_VIRTUAL = 4
MAX_CLASSES = 1024
MAX_FEATURES = 65536

STATUS_NAMES = {
    1: "CT_ERR_ARG", 2: "CT_ERR_OOM", 3: "CT_ERR_CUDA", 4: "CT_ERR_TIMEOUT",
    5: "CT_ERR_UNSUPPORTED", 6: "CT_ERR_INTERNAL", 7: "CT_ERR_CAPACITY",
}


class CudaTreeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Problem(C.Structure):
    _fields_ = [
        ("x_fm", C.c_void_p), ("labels", C.c_void_p), ("presort", C.c_void_p),
        ("n_rows", C.c_uint32), ("n_features", C.c_uint32), ("n_classes", C.c_uint32),
        ("index_bytes", C.c_uint32), ("label_bytes", C.c_uint32), ("max_features", C.c_uint32),
        ("min_samples_split", C.c_uint32), ("bootstrap", C.c_uint32), ("seed", C.c_uint64),
    ]


class Lists(C.Structure):
    _fields_ = [("si0", C.c_void_p), ("si1", C.c_void_p), ("mark", C.c_void_p),
                ("stride", C.c_uint32), ("n_slots", C.c_uint32)]


class Node(C.Structure):
    _fields_ = [("slot", C.c_uint32), ("start", C.c_uint32), ("n", C.c_uint32), ("raw_id", C.c_uint32),
                ("key", C.c_uint64), ("impurity", C.c_float), ("buf", C.c_uint32)]


class SplitResult(C.Structure):
    _fields_ = [("score", C.c_double), ("feature", C.c_uint32), ("pos", C.c_uint32),
                ("imp_left", C.c_float), ("imp_right", C.c_float), ("threshold", C.c_float),
                ("n_selected", C.c_uint32)]


class TreeBuffers(C.Structure):
    _fields_ = [("left", C.c_void_p), ("right", C.c_void_p), ("feature", C.c_void_p),
                ("threshold", C.c_void_p), ("value", C.c_void_p), ("n_nodes", C.c_void_p),
                ("capacity", C.c_uint32)]


class FitOptions(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("bfs_threshold", C.c_uint32), ("subtree_cutoff", C.c_uint32),
                ("scan_piece", C.c_uint32), ("flags", C.c_uint32), ("step_nodes", C.c_uint32),
                ("graph_samples", C.c_uint32), ("part_shape", C.c_uint32), ("huge_rows", C.c_uint32),
                ("small_rows", C.c_uint32)]


class FitJob(C.Structure):
    """ct_fit_job: one forest of a queue fit (ct_fit_queue)."""
    _fields_ = [("problem", Problem), ("lists", Lists), ("n_trees", C.c_uint32), ("first_tree", C.c_uint32)]


class PackedNode(C.Structure):
    _fields_ = [("threshold", C.c_float), ("feature", C.c_uint32), ("left", C.c_uint32),
                ("value", C.c_uint32)]


class KernelStats(C.Structure):
    _fields_ = [("launches", C.c_uint64 * 8), ("ms", C.c_double * 8), ("bytes", C.c_double * 8),
                ("steps", C.c_uint64), ("total_launches", C.c_uint64)]


KERNEL_GROUPS = ["select", "scan", "reduce", "mark", "partition", "children", "bootstrap", "subtree"]


def fit_stats() -> dict:
    """Per-kernel-group statistics of the last ct_fit on this thread."""
    st = KernelStats()
    call("ct_fit_stats", C.byref(st))
    return {"launches": list(st.launches), "ms": list(st.ms), "bytes": list(st.bytes),
            "steps": int(st.steps), "total_launches": int(st.total_launches)}


NODE_DTYPE_FIELDS = [("slot", "<u4"), ("start", "<u4"), ("n", "<u4"), ("raw_id", "<u4"),
                     ("key", "<u8"), ("impurity", "<f4"), ("buf", "<u4")]
SPLIT_DTYPE_FIELDS = [("score", "<f8"), ("feature", "<u4"), ("pos", "<u4"), ("imp_left", "<f4"),
                      ("imp_right", "<f4"), ("threshold", "<f4"), ("n_selected", "<u4")]

P = C.c_void_p
PROTOTYPES = {
    "ct_version": (C.c_char_p, []),
    "ct_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "ct_mark_bytes": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_size_t)]),
    "ct_presort_workspace_size": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_size_t)]),
    "ct_presort": (C.c_int, [P, C.c_uint32, C.c_uint32, C.c_uint32, P, P, C.c_size_t, P]),
    "ct_bootstrap_workspace_size": (C.c_int, [C.POINTER(Problem), C.POINTER(C.c_size_t)]),
    "ct_bootstrap_compact": (C.c_int, [C.POINTER(Problem), C.POINTER(Lists), C.c_uint32, C.c_uint32, P, P,
                                       C.c_size_t, P]),
    "ct_split_workspace_size": (C.c_int, [C.POINTER(Problem), C.c_uint32, C.c_uint64,
                                          C.POINTER(C.c_size_t)]),
    "ct_split_nodes": (C.c_int, [C.POINTER(Problem), C.POINTER(Lists), P, P, C.c_uint32, P, P, P,
                                 C.c_size_t, P]),
    "ct_split_nodes_noalloc": (C.c_int, [C.POINTER(Problem), C.POINTER(Lists), P, P, C.c_uint32, C.c_uint64,
                                         P, P]),
    "ct_partition_workspace_size": (C.c_int, [C.POINTER(Problem), C.c_uint32, C.c_uint64,
                                              C.POINTER(C.c_size_t)]),
    "ct_partition_nodes": (C.c_int, [C.POINTER(Problem), C.POINTER(Lists), P, P, C.c_uint32, P,
                                     C.c_size_t, P]),
    "ct_fit_workspace_size": (C.c_int, [C.POINTER(Problem), C.c_uint32, C.POINTER(FitOptions),
                                        C.POINTER(C.c_size_t)]),
    "ct_fit": (C.c_int, [C.POINTER(Problem), C.POINTER(Lists), C.c_uint32, C.c_uint32,
                         C.POINTER(FitOptions), C.POINTER(TreeBuffers), P, C.c_size_t, P]),
    "ct_fit_queue_workspace_size": (C.c_int, [C.POINTER(FitJob), C.c_uint32, C.POINTER(FitOptions),
                                              C.POINTER(C.c_size_t)]),
    "ct_fit_queue": (C.c_int, [C.POINTER(FitJob), C.c_uint32, C.POINTER(FitOptions), C.POINTER(TreeBuffers), P,
                               C.c_size_t, P]),
    "ct_fit_stats": (C.c_int, [C.c_void_p]),
    "ct_tree_canonicalize": (C.c_int, [P, P, P, P, P, C.c_uint32, P, P, P, P, P]),
    "ct_predict": (C.c_int, [P, C.c_uint32, P, C.c_uint32, P, C.c_uint32, C.c_uint32, C.c_uint32, P, P, P]),
    "ct_autotune_workspace_size": (C.c_int, [P, C.c_uint32, C.c_uint32, P]),
    "ct_autotune": (C.c_int, [P, P, C.c_uint32, C.c_uint32, P, P, C.c_size_t, P, P, P]),
    "ct_transpose_rows": (C.c_int, [P, C.c_uint32, C.c_uint32, P, P, P]),
    "ct_fetch_trees_scratch": (C.c_size_t, [C.c_uint64, C.c_uint32]),
    "ct_fetch_trees": (C.c_int, [P, C.c_uint32, P, P, C.c_size_t, P, P, P, P, P, P]),
    "ct_check_forest": (C.c_int, [P, C.c_uint32, P, C.c_uint32, C.c_uint32, C.c_uint32]),
    "ct_compact_fits": (C.c_int, [C.c_uint32, C.c_uint32]),
    "ct_compact_forest": (C.c_int, [P, C.c_uint32, C.c_uint32, C.c_uint32, P, P]),
    "ct_predict_compact": (C.c_int, [P, C.c_uint32, P, C.c_uint32, P, C.c_uint32, C.c_uint32, C.c_uint32, P, P,
                                     P]),
    "ct_server_create": (C.c_int, [P, P]),
    "ct_server_destroy": (C.c_int, [P]),
    "ct_server_add_forest": (C.c_int, [P, P, C.c_uint32, P, C.c_uint32, C.c_uint32, C.c_uint32, P]),
    "ct_server_remove_forest": (C.c_int, [P, C.c_uint32]),
    "ct_server_forest_info": (C.c_int, [P, C.c_uint32, P, P, P, P]),
    "ct_server_read_forest": (C.c_int, [P, C.c_uint32, P, P]),
    "ct_server_submit": (C.c_int, [P, P]),
    "ct_server_wait": (C.c_int, [P, P, C.c_double]),
    "ct_server_replay": (C.c_int, [P, P, C.c_uint32, C.c_double, P]),
    "ct_server_get_stats": (C.c_int, [P, P]),
}

_lib = None


def load() -> C.CDLL:
    """Load the shared library (once) and attach prototypes; raise if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH.name} is not built; run `python -m cudatree_b200.build` "
            "(this package has no CPU fallback)")
    lib = C.CDLL(os.fspath(LIB_PATH))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(1024)
    lib.ct_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != CT_OK:
        raise CudaTreeError(status, last_error())


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))


def mark_bytes(n_rows: int, n_slots: int) -> int:
    out = C.c_size_t()
    call("ct_mark_bytes", n_rows, n_slots, C.byref(out))
    return out.value


def version() -> str:
    return load().ct_version().decode()
