"""Many independent planning problems per launch (gprm_batch_* of the C ABI).

``ProblemBatch`` groups initialised ``RobotConfigspace`` handles of one
device - different robots, DOF, obstacle sets and dq - and checks the
configurations or edges of all of them in one persistent launch.  The
reference has no counterpart: it holds one scene per RobotConfigspace and
launches once per request (prm/src/lib/robotspace/robotconfigspace.cpp:
687-693).

Inputs are (rows, stride) float32 CUDA tensors, joint j of item i at
[j, i]; problem p owns items offsets[p] .. offsets[p+1]-1 and reads rows
0 .. ndof_p-1.  ``pack_items`` builds such an array from per-problem
(n_p, ndof_p) arrays.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _abi
from ._abi import Stats
from .configspace import GprmError, RobotConfigspace, _current_stream

MAX_DOF = 7
CONFIGS = 1
EDGES = 0


def offsets_of(counts: Sequence[int]) -> np.ndarray:
    return np.concatenate([[0], np.cumsum(np.asarray(counts, np.int64))]).astype(np.int64)


def pack_items(arrays: Sequence[np.ndarray], rows: int = MAX_DOF) -> tuple[np.ndarray, np.ndarray]:
    """[(n_p, ndof_p)] -> ((rows, total) float32 SoA, offsets (count+1,))."""
    offs = offsets_of([a.shape[0] for a in arrays])
    out = np.zeros((rows, int(offs[-1])), np.float32)
    for p, a in enumerate(arrays):
        out[:a.shape[1], offs[p]:offs[p + 1]] = np.asarray(a, np.float32).T
    return out, offs


class ProblemBatch:
    def __init__(self, spaces: Sequence[RobotConfigspace]):
        self.lib = _abi.load_library()
        self.spaces = list(spaces)   # keeps the handles alive while the batch lives
        arr = (C.c_void_p * len(self.spaces))(*[s.h.value for s in self.spaces])
        h = C.c_void_p()
        st = self.lib.gprm_batch_create(C.cast(arr, C.POINTER(C.c_void_p)), len(self.spaces), C.byref(h))
        if st != 0:
            raise GprmError(st, self.lib.gprm_batch_last_error(None).decode())
        self.h = h
        self.offsets = {CONFIGS: None, EDGES: None}

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.gprm_batch_destroy(h)
            self.h = None

    def _check(self, st: int):
        if st != 0:
            raise GprmError(st, self.lib.gprm_batch_last_error(self.h).decode())

    def set_layout(self, kind: int, offsets, queue_capacity: int = 0) -> None:
        offs = np.ascontiguousarray(offsets, np.int64)
        if offs.shape != (len(self.spaces) + 1,):
            raise ValueError(f"offsets must have {len(self.spaces) + 1} entries")
        self._check(self.lib.gprm_batch_set_layout(self.h, int(kind), offs.ctypes.data_as(C.POINTER(C.c_longlong)),
                                                   int(queue_capacity)))
        self.offsets[kind] = offs

    def check_configs_device(self, q, res, stream=None) -> None:
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_batch_indicator_device(self.h, C.c_void_p(q.data_ptr()),
                                                         C.c_void_p(res.data_ptr()), int(q.shape[1]),
                                                         C.c_void_p(st)))

    def check_edges_device(self, qs, qe, res, stream=None) -> None:
        assert qs.shape == qe.shape
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_batch_indicator2_device(self.h, C.c_void_p(qs.data_ptr()),
                                                          C.c_void_p(qe.data_ptr()), C.c_void_p(res.data_ptr()),
                                                          int(qs.shape[1]), C.c_void_p(st)))

    def capture(self, kind: int, qa, qb, res) -> None:
        self._check(self.lib.gprm_batch_capture(self.h, int(kind), C.c_void_p(qa.data_ptr()),
                                                C.c_void_p(qb.data_ptr() if qb is not None else 0),
                                                C.c_void_p(res.data_ptr()), int(qa.shape[1])))

    def replay(self, kind: int, stream=None) -> None:
        st = stream if stream is not None else _current_stream()
        self._check(self.lib.gprm_batch_replay(self.h, int(kind), C.c_void_p(st)))

    def set_launch(self, kind: int, threads: int, blocks_per_sm: int = 0) -> None:
        """Threads per block and at most blocks_per_sm resident blocks per
        SM (0: as many as fit)."""
        self._check(self.lib.gprm_batch_set_launch_shape(self.h, int(kind), int(threads), int(blocks_per_sm)))

    def get_launch(self, kind: int) -> dict:
        t, b, w = C.c_int(0), C.c_int(0), C.c_int(0)
        self._check(self.lib.gprm_batch_get_launch_shape(self.h, int(kind), C.byref(t), C.byref(b), C.byref(w)))
        return {"threads": t.value, "blocks_per_sm": b.value, "warps_per_sm": w.value}

    def autotune(self, kind: int, qa, qb, res, reps: int = 3) -> dict:
        """Times the launch shapes on this input and keeps the fastest;
        returns its shape and time per run (ms)."""
        t, ms = C.c_int(0), C.c_float(0)
        self._check(self.lib.gprm_batch_autotune(self.h, int(kind), C.c_void_p(qa.data_ptr()),
                                                 C.c_void_p(qb.data_ptr() if qb is not None else 0),
                                                 C.c_void_p(res.data_ptr()), int(qa.shape[1]), int(reps),
                                                 C.byref(t), C.byref(ms)))
        return dict(self.get_launch(kind), ms=ms.value, solo=self.get_solo_threshold(kind))

    def tune_table(self, kind: int) -> list:
        """The last autotune's candidates: [{threads, blocks_per_sm, ms}]."""
        import numpy as np
        cnt = C.c_int(0)
        self._check(self.lib.gprm_batch_get_tune_table(self.h, int(kind), 0, None, None, None, None, C.byref(cnt)))
        n = cnt.value
        t, b, ms = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.float32)
        so = np.zeros(n, np.int64)
        if n:
            self._check(self.lib.gprm_batch_get_tune_table(self.h, int(kind), n, t.ctypes.data, b.ctypes.data,
                                                           so.ctypes.data, ms.ctypes.data, C.byref(cnt)))
        return [{"threads": int(t[i]), "blocks_per_sm": int(b[i]), "solo_min_items": int(so[i]), "ms": float(ms[i])}
                for i in range(n)]

    def set_solo_threshold(self, kind: int, min_items: int) -> None:
        """Problems with at least min_items items run in their own launches
        (-1: none, 0: all); drops the kind's captured graph."""
        self._check(self.lib.gprm_batch_set_solo_threshold(self.h, int(kind), int(min_items)))

    def get_solo_threshold(self, kind: int) -> dict:
        m, n = C.c_longlong(0), C.c_int(0)
        self._check(self.lib.gprm_batch_get_solo_threshold(self.h, int(kind), C.byref(m), C.byref(n)))
        return {"min_items": m.value, "solo_problems": n.value}

    def stats(self) -> dict:
        s = Stats()
        self._check(self.lib.gprm_batch_get_stats(self.h, C.byref(s)))
        return {name: int(getattr(s, name)) for name, _ in Stats._fields_}
