"""Helpers for the GPU tests: build problems and node lists, call the C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from cudatree_b200 import _lib
from oracle import cudatree_oracle as O


def dev():
    return torch.device("cuda", 0)


def to_dev(a: np.ndarray) -> torch.Tensor:
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(dev())


def dev_bytes(n: int) -> torch.Tensor:
    # +64: index buffers are read up to 15 bytes past their end by 16-byte bulk copies
    return torch.zeros(max(int(n), 1) + 64, dtype=torch.uint8, device=dev())


def from_dev(t: torch.Tensor, dtype, shape=None) -> np.ndarray:
    a = t.cpu().numpy().view(dtype)
    return a.reshape(shape) if shape is not None else a


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class GpuProblem:
    """Device copies of (x, y) + presort, and the ct_problem struct."""

    def __init__(self, x: np.ndarray, y: np.ndarray, n_classes: int, max_features: int,
                 min_samples_split: int = 1, bootstrap: bool = False, seed: int = 0,
                 index_bytes: int | None = None):
        self.x = np.ascontiguousarray(x, dtype=np.float32)
        self.y = np.asarray(y, dtype=np.int64)
        self.n, self.f = self.x.shape
        self.c = int(n_classes)
        self.ib = index_bytes or (2 if self.n <= 0xFFFF else 4)
        self.lb = 1 if self.c <= 255 else 2
        self.idx_dtype = np.uint16 if self.ib == 2 else np.uint32
        self.x_fm_np = np.ascontiguousarray(self.x.T)
        self.x_fm = to_dev(self.x_fm_np)
        self.labels = to_dev(self.y.astype(np.uint8 if self.lb == 1 else np.uint16))
        self.presort = dev_bytes(self.f * self.n * self.ib)
        ws = C.c_size_t()
        _lib.call("ct_presort_workspace_size", self.n, self.f, C.byref(ws))
        pws = dev_bytes(ws.value)
        _lib.call("ct_presort", self.x_fm.data_ptr(), self.n, self.f, self.ib, self.presort.data_ptr(),
                  pws.data_ptr(), ws.value, stream())
        self.prob = _lib.Problem(self.x_fm.data_ptr(), self.labels.data_ptr(), self.presort.data_ptr(),
                                 self.n, self.f, self.c, self.ib, self.lb, max_features,
                                 min_samples_split, int(bootstrap), seed)

    def presort_np(self) -> np.ndarray:
        nb = self.f * self.n * self.ib
        return from_dev(self.presort[:nb], self.idx_dtype, (self.f, self.n)).astype(np.int64)


class GpuLists:
    def __init__(self, gp: GpuProblem, slots: int = 1):
        self.gp = gp
        self.slots = slots
        nbytes = slots * gp.f * gp.n * gp.ib
        self.si = [dev_bytes(nbytes), dev_bytes(nbytes)]
        self.mark = dev_bytes(_lib.mark_bytes(gp.n, slots))
        self.lists = _lib.Lists(self.si[0].data_ptr(), self.si[1].data_ptr(), self.mark.data_ptr(), gp.n,
                                slots)

    def get(self, buf: int, slot: int = 0) -> np.ndarray:
        gp = self.gp
        nb = self.slots * gp.f * gp.n * gp.ib
        a = from_dev(self.si[buf][:nb], gp.idx_dtype, (self.slots, gp.f, gp.n))
        return a[slot].astype(np.int64)

    def put(self, buf: int, lists: np.ndarray, slot: int = 0) -> None:
        gp = self.gp
        nb = self.slots * gp.f * gp.n * gp.ib
        a = from_dev(self.si[buf][:nb], gp.idx_dtype, (self.slots, gp.f, gp.n)).copy()
        a[slot] = lists.astype(gp.idx_dtype)
        self.si[buf][:nb].copy_(to_dev(a))


def node_array(nodes: list[dict]) -> np.ndarray:
    dt = np.dtype(_lib.NODE_DTYPE_FIELDS)
    a = np.zeros(len(nodes), dtype=dt)
    for i, nd in enumerate(nodes):
        for k, v in nd.items():
            a[i][k] = v
    return a


def split_nodes(gp: GpuProblem, gl: GpuLists, nodes: np.ndarray, totals: np.ndarray):
    nn = nodes.shape[0]
    total = int(nodes["n"].sum())
    ws = C.c_size_t()
    _lib.call("ct_split_workspace_size", C.byref(gp.prob), nn, total, C.byref(ws))
    work = dev_bytes(ws.value)
    nd = to_dev(nodes)
    td = to_dev(totals.astype(np.uint32))
    out = dev_bytes(nn * 32)
    sel = dev_bytes(nn * gp.prob.max_features * 4)
    _lib.call("ct_split_nodes", C.byref(gp.prob), C.byref(gl.lists), nd.data_ptr(), td.data_ptr(), nn,
              out.data_ptr(), sel.data_ptr(), work.data_ptr(), ws.value, stream())
    res = from_dev(out[:nn * 32], np.dtype(_lib.SPLIT_DTYPE_FIELDS))
    sel_np = from_dev(sel[:nn * gp.prob.max_features * 4], np.uint32, (nn, gp.prob.max_features))
    return res, sel_np, out


def partition_nodes(gp: GpuProblem, gl: GpuLists, nodes: np.ndarray, results_dev: torch.Tensor):
    nn = nodes.shape[0]
    total = int(nodes["n"].sum())
    ws = C.c_size_t()
    _lib.call("ct_partition_workspace_size", C.byref(gp.prob), nn, total, C.byref(ws))
    work = dev_bytes(ws.value)
    nd = to_dev(nodes)
    _lib.call("ct_partition_nodes", C.byref(gp.prob), C.byref(gl.lists), nd.data_ptr(),
              results_dev.data_ptr(), nn, work.data_ptr(), ws.value, stream())
    torch.cuda.synchronize()


def grouped_lists(x_fm: np.ndarray, groups: list[np.ndarray]) -> tuple[np.ndarray, list[int]]:
    """Feature lists where each group of rows is one node range sorted by (x, row)."""
    f, n = x_fm.shape
    lists = np.zeros((f, n), dtype=np.int64)
    starts = []
    pos = 0
    for g in groups:
        starts.append(pos)
        for j in range(f):
            order, _ = O.node_sorted(x_fm, j, g)
            lists[j, pos:pos + g.shape[0]] = g[order]
        pos += g.shape[0]
    return lists, starts
