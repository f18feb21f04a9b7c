"""Python mirror of the reference's collision-checker interface.

``RobotConfigspace`` follows ``Configspace<ndof>`` / ``RobotConfigspace<ndof>``
(prm/src/lib/prm/configspace.hpp:10-50, prm/src/lib/robotspace/
robotconfigspace.h:25-176): same method names, argument meanings, layouts
(q[i + offset*j]) and verdict codes, over the C ABI of libgprm_b200.so.
Failures raise ``GprmError`` carrying the library's message (the reference
asserted instead).  There is no CPU fallback: without the CUDA library the
constructor raises.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from ._abi import DescHolder, Stats, fptr, iptr


class GprmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gprm status {status}: {message}")
        self.status = status


def _check(lib, h, status: int):
    if status != 0:
        msg = lib.gprm_last_error(h)
        raise GprmError(status, msg.decode() if msg else "")


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, np.float32))


def _soa_offset(t) -> int:
    """Row stride (the C ABI's offset) of an (ndof, n) SoA tensor whose
    columns are contiguous."""
    if t.dim() != 2 or (t.shape[1] > 1 and t.stride(1) != 1):
        raise ValueError("expected an (ndof, n) tensor with unit column stride")
    return int(t.stride(0)) if t.shape[0] > 1 else int(t.shape[1])


class RobotConfigspace:
    """One scene on one GPU.

    ``RobotConfigspace(scene, dq, nbuf)`` takes a ``scenes.Scene``;
    ``RobotConfigspace(path, dq, nbuf, ndof=...)`` reads the reference's config
    directory (robotconfigspace.cpp:84-98).  ``nbuf`` bounds the edges of one
    indicator2 call like the reference (0 = unbounded).
    """

    def __init__(self, scene_or_path, dq: float = 0.01, nbuf: int = 0, ndof: Optional[int] = None):
        self.lib = _abi.load_library()
        h = C.c_void_p()
        if isinstance(scene_or_path, str):
            if ndof is None:
                ndof = int(np.fromfile(scene_or_path + "/ndof.bin", np.int32)[0])
            st = self.lib.gprm_create_from_dir(scene_or_path.encode(), int(ndof), float(dq), int(nbuf),
                                               C.byref(h))
        else:
            self._desc = DescHolder(scene_or_path)
            st = self.lib.gprm_create(self._desc.ref(), float(dq), int(nbuf), C.byref(h))
        _check(self.lib, None, st)
        self.h = h
        self._ndof = self.lib.gprm_dim(h)
        self._pending = {}

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.gprm_destroy(h)
            self.h = None

    # -- lifetime / options ------------------------------------------------
    def init(self, rank: int = 0, size: int = 1) -> int:
        _check(self.lib, self.h, self.lib.gprm_init(self.h, rank, size))
        return 0

    def set_mode(self, mode: int) -> None:
        _check(self.lib, self.h, self.lib.gprm_set_mode(self.h, mode))

    def set_edge_policy(self, policy: int) -> None:
        _check(self.lib, self.h, self.lib.gprm_set_edge_policy(self.h, policy))

    def set_edge_split(self, max_edges: int, seg_rounds: int = 2) -> None:
        """Edge batches of at most max_edges (<= 2^22; 0 = never) split edges
        longer than seg_rounds x 32 steps over several warps (same codes)."""
        _check(self.lib, self.h, self.lib.gprm_set_edge_split(self.h, max_edges, seg_rounds))

    def set_band(self, band_m: float) -> None:
        _check(self.lib, self.h, self.lib.gprm_set_band(self.h, band_m))

    def stats(self) -> dict:
        s = Stats()
        _check(self.lib, self.h, self.lib.gprm_get_stats(self.h, C.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in Stats._fields_}

    # -- Configspace<ndof> -------------------------------------------------
    def indicator(self, q, res=None, N: Optional[int] = None, offset: Optional[int] = None):
        """indicator(q) -> code for one configuration q[ndof]; or the batched
        indicator(q, res, N, offset) filling res[i] for q[i + offset*j]."""
        if res is None:
            qq = _f32(q).reshape(-1)
            assert qq.size == self._ndof
            code = C.c_int(0)
            _check(self.lib, self.h, self.lib.gprm_indicator(self.h, fptr(qq), C.byref(code)))
            return code.value
        qq = _f32(q)
        assert res.dtype == np.int32 and res.flags.c_contiguous
        _check(self.lib, self.h, self.lib.gprm_indicator_batch(self.h, fptr(qq), iptr(res), int(N), int(offset)))
        return 0

    def indicator2(self, qs, qe, res: np.ndarray, N: int, offset: int) -> int:
        a, b = _f32(qs), _f32(qe)
        assert res.dtype == np.int32 and res.flags.c_contiguous
        _check(self.lib, self.h, self.lib.gprm_indicator2(self.h, fptr(a), fptr(b), iptr(res), int(N), int(offset)))
        return 0

    def indicator2_async(self, qs, qe, res: np.ndarray, N: int, offset: int) -> int:
        a, b = _f32(qs), _f32(qe)
        assert res.dtype == np.int32 and res.flags.c_contiguous
        req = C.c_int(0)
        _check(self.lib, self.h, self.lib.gprm_indicator2_async(self.h, fptr(a), fptr(b), iptr(res), int(N),
                                                                 int(offset), C.byref(req)))
        self._pending[req.value] = (a, b, res)  # keep buffers alive until wait
        return req.value

    def indicator2_async_wait(self, request: int) -> int:
        try:
            _check(self.lib, self.h, self.lib.gprm_indicator2_wait(self.h, int(request)))
        finally:
            self._pending.pop(request, None)
        return 0

    def check_boundaries(self, q, res=None, N: Optional[int] = None, offset: Optional[int] = None):
        if res is None:
            qq = _f32(q).reshape(-1)
            out = C.c_int(0)
            _check(self.lib, self.h, self.lib.gprm_check_boundaries1(self.h, fptr(qq), C.byref(out)))
            return out.value
        qq = _f32(q)
        _check(self.lib, self.h, self.lib.gprm_check_boundaries(self.h, fptr(qq), iptr(res), int(N), int(offset)))
        return 0

    def min(self, i: int) -> float:
        return float(self.lib.gprm_min(self.h, i))

    def max(self, i: int) -> float:
        return float(self.lib.gprm_max(self.h, i))

    def deltaq(self) -> float:
        return float(self.lib.gprm_deltaq(self.h))

    def dim(self) -> int:
        return self._ndof

    # -- numpy conveniences (n, ndof) arrays ----------------------------------
    def check_configs(self, q: np.ndarray) -> np.ndarray:
        q = _f32(q)
        n = q.shape[0]
        buf = np.ascontiguousarray(q.T).reshape(-1)
        res = np.zeros(n, np.int32)
        self.indicator(buf, res, n, n)
        return res

    def check_edges(self, qs: np.ndarray, qe: np.ndarray) -> np.ndarray:
        qs, qe = _f32(qs), _f32(qe)
        n = qs.shape[0]
        a = np.ascontiguousarray(qs.T).reshape(-1)
        b = np.ascontiguousarray(qe.T).reshape(-1)
        res = np.zeros(n, np.int32)
        self.indicator2(a, b, res, n, n)
        return res

    # -- device buffers (torch tensors, SoA (ndof, n) float32 on the GPU) --------
    def indicator2_compressed(self, qs, M: int, qe, res, posqe, numqe, offset: int) -> int:
        """indicator2(qs, M, qe, res, posqe, numqe, offset): res[l] for the
        edges qs[k] -> qe[l], l in posqe[k] .. posqe[k]+numqe[k]-1 (qs SoA
        with row stride M, qe with row stride offset; host arrays)."""
        a, b = _f32(qs), _f32(qe)
        assert res.dtype == np.int32 and res.flags.c_contiguous
        pos = np.ascontiguousarray(posqe, np.int32)
        num = np.ascontiguousarray(numqe, np.int32)
        _check(self.lib, self.h, self.lib.gprm_indicator2_compressed(self.h, fptr(a), int(M), fptr(b), iptr(res),
                                                                    iptr(pos), iptr(num), int(offset)))
        return 0

    def check_configs_device(self, q_soa, res, stream=None) -> None:
        """q_soa: (ndof, n) float32 CUDA tensor with unit column stride
        (a column slice of a wider SoA array works: its row stride is the
        offset); res: (n,) int32."""
        n = int(q_soa.shape[1])
        off = _soa_offset(q_soa)
        st = stream if stream is not None else _current_stream()
        _check(self.lib, self.h, self.lib.gprm_indicator_batch_device(
            self.h, C.c_void_p(q_soa.data_ptr()), C.c_void_p(res.data_ptr()), n, off, C.c_void_p(st)))

    def check_edges_device(self, qs_soa, qe_soa, res, stream=None) -> None:
        """qs_soa, qe_soa: (ndof, n) float32 CUDA tensors of one row stride
        (as check_configs_device); res: (n,) int32."""
        n = int(qs_soa.shape[1])
        off = _soa_offset(qs_soa)
        if _soa_offset(qe_soa) != off:
            raise ValueError("qs and qe must have the same row stride")
        st = stream if stream is not None else _current_stream()
        _check(self.lib, self.h, self.lib.gprm_indicator2_device(
            self.h, C.c_void_p(qs_soa.data_ptr()), C.c_void_p(qe_soa.data_ptr()), C.c_void_p(res.data_ptr()),
            n, off, C.c_void_p(st)))

    def set_launch(self, vertex_kernel: bool, threads: int, scene_in_smem: bool, blocks_per_sm: int = 0) -> None:
        """Launch shape of the FP32 kernels: threads per block, scene table in
        shared memory or through L1, and at most blocks_per_sm resident
        blocks per SM (0: as many as fit; fewer leave more L1)."""
        _check(self.lib, self.h, self.lib.gprm_set_launch_shape(self.h, int(vertex_kernel), threads,
                                                                int(scene_in_smem), int(blocks_per_sm)))

    def get_launch(self, vertex_kernel: bool) -> dict:
        t, s, w = C.c_int(0), C.c_int(0), C.c_int(0)
        _check(self.lib, self.h, self.lib.gprm_get_launch(self.h, int(vertex_kernel), C.byref(t), C.byref(s), C.byref(w)))
        return {"threads": t.value, "scene_in_smem": bool(s.value), "warps_per_sm": w.value}

    def profile_enable(self, on: bool = True) -> None:
        _check(self.lib, self.h, self.lib.gprm_profile_enable(self.h, 1 if on else 0))

    def profile_read(self) -> dict:
        a, b, n = C.c_double(0), C.c_double(0), C.c_int64(0)
        _check(self.lib, self.h, self.lib.gprm_profile_read(self.h, C.byref(a), C.byref(b), C.byref(n)))
        return {"fp32_ms": a.value, "fp64_ms": b.value, "fp32_launches": int(n.value)}

    def debug_fk(self, q) -> np.ndarray:
        qq = _f32(q).reshape(-1)
        out = np.zeros((self._ndof + 1) * 12, np.float32)
        _check(self.lib, self.h, self.lib.gprm_debug_fk(self.h, fptr(qq), fptr(out)))
        return out.reshape(self._ndof + 1, 4, 3)


def measure_fp32_peak() -> float:
    """FP32 FMA throughput of the current device, TFLOP/s."""
    lib = _abi.load_library()
    t = C.c_double(0)
    st = lib.gprm_measure_fp32_peak(C.byref(t))
    if st != 0:
        raise GprmError(st, "fp32 peak probe failed")
    return t.value


def _current_stream() -> int:
    import torch
    return int(torch.cuda.current_stream().cuda_stream)
