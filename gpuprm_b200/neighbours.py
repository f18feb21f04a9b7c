"""Neighbour search on the device (gprm_nbr_* of the C ABI).

``NeighbourIndex`` indexes roadmap nodes held as a (ndof, n) float32 CUDA
tensor and answers radius queries with the reference's get_near_vertices
arithmetic (prm/src/lib/prm/prmsolver.cpp:2533-2574) and exact k-nearest
queries under the same distance.
"""
from __future__ import annotations

import ctypes as C

from . import _abi
from .configspace import GprmError, _current_stream


class NeighbourIndex:
    def __init__(self, ndof: int):
        self.lib = _abi.load_library()
        h = C.c_void_p()
        st = self.lib.gprm_nbr_create(int(ndof), C.byref(h))
        if st != 0:
            raise GprmError(st, self.lib.gprm_nbr_last_error(None).decode())
        self.h = h
        self.ndof = ndof
        self.nodes = None

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.gprm_nbr_destroy(h)
            self.h = None

    def _check(self, st):
        if st != 0:
            raise GprmError(st, self.lib.gprm_nbr_last_error(self.h).decode())

    def build(self, x, cell: float = 0.0, stream=None) -> None:
        """x: (ndof, n) contiguous float32 CUDA tensor, kept referenced."""
        assert x.shape[0] == self.ndof and x.is_contiguous()
        self.nodes = x
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_nbr_build(self.h, C.c_void_p(x.data_ptr()), int(x.shape[1]), int(x.shape[1]),
                                            float(cell), C.c_void_p(st)))

    def radius(self, q, D: float, cap: int, stream=None):
        """q: (ndof, m) -> (counts (m,), idx (m, cap), dist (m, cap))."""
        import torch
        m = int(q.shape[1])
        counts = torch.empty(m, dtype=torch.int32, device=q.device)
        idx = torch.full((m, cap), -1, dtype=torch.int32, device=q.device)
        dist = torch.full((m, cap), float("inf"), dtype=torch.float32, device=q.device)
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_nbr_radius(self.h, C.c_void_p(q.data_ptr()), m, m, float(D), int(cap),
                                             C.c_void_p(counts.data_ptr()), C.c_void_p(idx.data_ptr()),
                                             C.c_void_p(dist.data_ptr()), C.c_void_p(st)))
        return counts, idx, dist

    def knn(self, k: int, q=None, stream=None):
        """k nearest nodes of every node (q None, the node itself excluded)
        or of the queries q (ndof, m) -> (idx (m, k), dist (m, k))."""
        import torch
        self_q = q is None
        m = int(self.nodes.shape[1]) if self_q else int(q.shape[1])
        dev = self.nodes.device
        idx = torch.empty((m, k), dtype=torch.int32, device=dev)
        dist = torch.empty((m, k), dtype=torch.float32, device=dev)
        st = stream if stream is not None else _current_stream()
        qp = 0 if self_q else q.data_ptr()
        self._check(self.lib.gprm_nbr_knn(self.h, C.c_void_p(qp), m, m, int(k), 1 if self_q else 0,
                                          C.c_void_p(idx.data_ptr()), C.c_void_p(dist.data_ptr()), C.c_void_p(st)))
        return idx, dist

    def redo_count(self) -> int:
        n = C.c_int(0)
        self._check(self.lib.gprm_nbr_redo_count(self.h, C.byref(n)))
        return n.value


def knn_pairs(q_soa, k: int):
    """Undirected k-nearest-neighbour pairs (i < j) of the columns of q_soa,
    a (ndof, n) float32 CUDA tensor; two int64 CUDA tensors."""
    import torch
    n = int(q_soa.shape[1])
    if n < 2:
        e = torch.empty(0, dtype=torch.int64, device=q_soa.device)
        return e, e
    index = NeighbourIndex(int(q_soa.shape[0]))
    index.build(q_soa.contiguous())
    idx, _ = index.knn(min(k, n - 1))
    rows = torch.arange(n, device=q_soa.device)[:, None].expand_as(idx)
    valid = idx >= 0
    i = rows[valid].to(torch.int64)
    j = idx[valid].to(torch.int64)
    a = torch.minimum(i, j)
    b = torch.maximum(i, j)
    key = torch.unique(a * n + b)
    return key // n, key % n
