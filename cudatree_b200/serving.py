"""Serving engine binding: resident forests, continuously batched predict
requests, small fit jobs, admission by an HBM budget, p50/p99 latency.

The engine lives in libcudatree_b200.so (``ct_server_*``); this module packs
fitted forests for it, builds request records, and maps predicted class ids
back to the forest's labels.  The reference has no serving path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .forest_queue import fit_forests  # noqa: F401  (the forest queue: shared level steps)
from .random_forest import PACKED_DTYPE, RandomForestClassifier, pack_trees, restore_forest, unpack_trees

CT_REQ_PREDICT = 0
CT_REQ_FIT = 1


class ServerConfig(C.Structure):
    _fields_ = [("max_batch_rows", C.c_uint32), ("max_features", C.c_uint32), ("small_rows", C.c_uint32),
                ("fit_workers", C.c_uint32), ("max_fit_rows", C.c_uint32), ("max_fit_trees", C.c_uint32),
                ("max_classes", C.c_uint32), ("reserved", C.c_uint32), ("hbm_budget_bytes", C.c_uint64),
                ("forest_pool_bytes", C.c_uint64)]


class Request(C.Structure):
    _fields_ = [("arrival_s", C.c_double), ("kind", C.c_uint32), ("forest", C.c_uint32),
                ("x", C.c_void_p), ("y", C.c_void_p), ("pred", C.c_void_p),
                ("n_rows", C.c_uint32), ("n_features", C.c_uint32), ("n_classes", C.c_uint32),
                ("n_trees", C.c_uint32), ("max_features", C.c_uint32), ("status", C.c_uint32),
                ("seed", C.c_uint64), ("latency_ms", C.c_double), ("result_forest", C.c_uint32),
                ("pad_", C.c_uint32), ("pending_", C.c_void_p)]


class ServerStats(C.Structure):
    _fields_ = [("requests", C.c_uint64), ("rows", C.c_uint64), ("batches", C.c_uint64),
                ("fit_jobs", C.c_uint64), ("rejected", C.c_uint64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("p50_small_ms", C.c_double),
                ("p99_small_ms", C.c_double), ("p50_fit_ms", C.c_double), ("p99_fit_ms", C.c_double),
                ("max_ms", C.c_double), ("wall_s", C.c_double), ("rows_per_s", C.c_double),
                ("hbm_used_bytes", C.c_uint64), ("hbm_budget_bytes", C.c_uint64),
                ("forest_bytes", C.c_uint64), ("forest_pool_bytes", C.c_uint64),
                ("zero_copy_requests", C.c_uint64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def _host_ptr(a) -> int:
    if isinstance(a, torch.Tensor):
        return a.data_ptr()
    if not (isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"]):
        raise ValueError("host arrays must be C-contiguous numpy arrays or torch tensors")
    return a.ctypes.data


def pinned(a: np.ndarray) -> torch.Tensor:
    """Page-locked host copy of an array (asynchronous copies need it)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.pin_memory()


class ForestServer:
    """Resident forests + request loop on the current CUDA device.  All of the
    server's device memory (staging, fit arenas, the forest pool) is taken at
    construction, inside hbm_budget_bytes."""

    def __init__(self, max_batch_rows=0, max_features=512, small_rows=4096, fit_workers=2,
                 max_fit_rows=20000, max_fit_trees=10, hbm_budget_bytes=0, max_classes=64, forest_pool_bytes=0):
        _lib.load()
        torch.cuda.init()
        cfg = ServerConfig(max_batch_rows, max_features, small_rows, fit_workers, max_fit_rows,
                           max_fit_trees, max_classes, 0, hbm_budget_bytes, forest_pool_bytes)
        h = C.c_void_p()
        _lib.call("ct_server_create", C.byref(cfg), C.byref(h))
        self._h = h
        self._tables = {}       # label table per forest id (fit jobs' forests use class ids)

    def close(self):
        if self._h:
            _lib.load().ct_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_forest(self, forest: RandomForestClassifier) -> int:
        packed, offsets = pack_trees(forest._trees)
        return self.add_packed(packed, offsets, forest.n_features, forest.n_labels, forest.compt_table)

    def add_packed(self, packed: np.ndarray, offsets: np.ndarray, n_features: int, n_classes: int,
                   table=None) -> int:
        packed = np.ascontiguousarray(packed, dtype=PACKED_DTYPE)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        fid = C.c_uint32()
        _lib.call("ct_server_add_forest", self._h, packed.ctypes.data, packed.shape[0], offsets.ctypes.data,
                  offsets.shape[0], n_features, n_classes, C.byref(fid))
        if table is not None:
            self._tables[fid.value] = np.asarray(table)
        return fid.value

    def load_forest(self, source) -> int:
        """Make a stored forest resident: source is a path or the bytes of the
        versioned flat format (forest_format), whose node section goes to the
        forest pool as it is, after the host check."""
        from . import forest_format
        if isinstance(source, (bytes, bytearray, memoryview)):
            data = bytes(source)
        else:
            with open(source, "rb") as fh:
                data = fh.read()
        packed, offsets, hdr, table = forest_format.decode(data)
        return self.add_packed(packed, offsets, hdr["n_features"], hdr["n_classes"], table)

    def read_forest(self, forest_id: int):
        """(packed nodes, tree offsets, n_features, n_classes) of a resident forest, exactly as added or fitted."""
        nn, nt, nf, nc = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        _lib.call("ct_server_forest_info", self._h, forest_id, C.byref(nn), C.byref(nt), C.byref(nf), C.byref(nc))
        packed = np.zeros(nn.value, dtype=PACKED_DTYPE)
        offsets = np.zeros(nt.value, dtype=np.uint32)
        _lib.call("ct_server_read_forest", self._h, forest_id, packed.ctypes.data, offsets.ctypes.data)
        return packed, offsets, nf.value, nc.value

    def forest(self, forest_id: int, table=None, params=None) -> RandomForestClassifier:
        """A RandomForestClassifier holding a copy of a resident forest's trees
        (table: the label of each class id; default: the forest's own table,
        else the class ids)."""
        packed, offsets, nf, nc = self.read_forest(forest_id)
        if table is None:
            table = self._tables.get(forest_id, np.arange(nc))
        dt = np.uint8 if nc <= 255 else np.uint16
        return restore_forest(unpack_trees(packed, offsets, nf, dt), np.dtype(dt).str, np.asarray(table), nf,
                              params)

    def remove_forest(self, forest_id: int) -> None:
        """Retire a forest; its pool bytes return when its launched batches complete."""
        _lib.call("ct_server_remove_forest", self._h, forest_id)
        self._tables.pop(forest_id, None)

    def predict_request(self, forest_id: int, x_pinned: torch.Tensor, out_pinned: torch.Tensor) -> Request:
        n = x_pinned.shape[0]
        return Request(0.0, CT_REQ_PREDICT, forest_id, x_pinned.data_ptr(), None, out_pinned.data_ptr(), n,
                       x_pinned.shape[1], 0, 0, 0, 0, 0, 0.0, 0, 0, None)

    def fit_request(self, x, y, n_classes: int, n_trees: int, seed: int, max_features: int = 0) -> Request:
        """A fit job over host arrays x [n, f] float32 and y [n] uint32 class ids
        (torch tensors or numpy arrays; pageable memory is fine for fit jobs,
        whose copies are staged by the fit worker's own thread)."""
        n, f = x.shape
        return Request(0.0, CT_REQ_FIT, 0, _host_ptr(x), _host_ptr(y), None, n, f, n_classes,
                       n_trees, max_features, 0, seed, 0.0, 0, 0, None)

    def submit(self, req: Request) -> None:
        _lib.call("ct_server_submit", self._h, C.byref(req))

    def wait(self, req: Request, timeout_s: float = 60.0) -> int:
        return _lib.load().ct_server_wait(self._h, C.byref(req), timeout_s)

    def predict(self, forest_id: int, x: np.ndarray) -> np.ndarray:
        """One predict request through the server; labels in the forest's label space."""
        xp = pinned(np.asarray(x, dtype=np.float32))
        out = torch.empty(xp.shape[0], dtype=torch.int32).pin_memory()
        req = self.predict_request(forest_id, xp, out)
        self.submit(req)
        _lib.check(self.wait(req))
        ids = out.numpy().astype(np.int64)
        table = self._tables.get(forest_id)
        return ids if table is None else table[ids]

    def replay(self, reqs, timeout_s: float = 120.0) -> dict:
        arr = (Request * len(reqs))(*reqs)
        st = ServerStats()
        _lib.call("ct_server_replay", self._h, arr, len(reqs), timeout_s, C.byref(st))
        for i, r in enumerate(reqs):  # copy results back into the caller's records
            C.memmove(C.addressof(r), C.addressof(arr[i]), C.sizeof(Request))
        return st.as_dict()

    def stats(self) -> dict:
        st = ServerStats()
        _lib.call("ct_server_get_stats", self._h, C.byref(st))
        return st.as_dict()
