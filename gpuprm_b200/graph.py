"""Roadmap graph operations on the device (gprm_graph_* of the C ABI).

Edge lists are int32 CUDA tensors (eu, ev) with an optional uint8 mask of
usable edges; see include/gprm_b200.h for the semantics (components by
union-find, breadth-first forests with deterministic parents, forest paths,
float single-source shortest paths equal to Dijkstra's).
"""
from __future__ import annotations

import ctypes as C

from . import _abi
from .configspace import GprmError, _current_stream


def _p(t):
    return C.c_void_p(t.data_ptr() if t is not None else 0)


class RoadmapGraph:
    def __init__(self):
        self.lib = _abi.load_library()
        h = C.c_void_p()
        st = self.lib.gprm_graph_create(C.byref(h))
        if st != 0:
            raise GprmError(st, self.lib.gprm_graph_last_error(None).decode())
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.gprm_graph_destroy(h)
            self.h = None

    def _check(self, st):
        if st != 0:
            raise GprmError(st, self.lib.gprm_graph_last_error(self.h).decode())

    def components(self, V: int, eu, ev, mask=None, stream=None):
        import torch
        label = torch.empty(V, dtype=torch.int32, device=eu.device)
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_graph_components(self.h, V, int(eu.numel()), _p(eu), _p(ev), _p(mask),
                                                   _p(label), C.c_void_p(st)))
        return label

    def forest(self, V: int, eu, ev, label, mask=None, stream=None):
        import torch
        parent = torch.empty(V, dtype=torch.int32, device=eu.device)
        depth = torch.empty(V, dtype=torch.int32, device=eu.device)
        levels = C.c_int(0)
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_graph_forest(self.h, V, int(eu.numel()), _p(eu), _p(ev), _p(mask), _p(label),
                                               _p(parent), _p(depth), C.byref(levels), C.c_void_p(st)))
        return parent, depth, levels.value

    def paths(self, qs, qt, label, parent, depth, stream=None):
        """Forest paths qs[t] -> qt[t]: (len (Q,), offsets (Q,), flat int32 vertex ids)."""
        import torch
        V = int(label.numel())
        Q = int(qs.numel())
        dev = qs.device
        length = torch.empty(Q, dtype=torch.int32, device=dev)
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_graph_path_lengths(self.h, V, Q, _p(qs), _p(qt), _p(label), _p(parent), _p(depth),
                                                     _p(length), C.c_void_p(st)))
        off = torch.cumsum(length.to(torch.int64), 0) - length.to(torch.int64)
        total = int((off[-1] + length[-1]).item()) if Q else 0
        flat = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
        self._check(self.lib.gprm_graph_path_write(self.h, Q, _p(qs), _p(qt), _p(parent), _p(depth), _p(length),
                                                   _p(off), _p(flat), C.c_void_p(st)))
        return length, off, flat[:total]

    def sssp(self, V: int, eu, ev, w, src: int, mask=None, stream=None):
        import torch
        dist = torch.empty(V, dtype=torch.float32, device=eu.device)
        parent = torch.empty(V, dtype=torch.int32, device=eu.device)
        rounds = C.c_int(0)
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_graph_sssp(self.h, V, int(eu.numel()), _p(eu), _p(ev), _p(mask), _p(w), int(src),
                                             _p(dist), _p(parent), C.byref(rounds), C.c_void_p(st)))
        return dist, parent, rounds.value
