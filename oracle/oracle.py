"""ctypes loader for the CPU oracle.

TEST INFRASTRUCTURE ONLY: used by tests/, by the smoke check and by the
bench's CPU-baseline leg, as the checker or the timed CPU reference.  The
product (gpuprm_b200) never imports this module.

* ``Oracle``      liboracle.so, the restatement in gprm_oracle.cpp
* ``RefChecker``  _ref/libgprm_ref.so, the reference's own CPU checker built
                  from its sources by oracle/Makefile (present only where
                  the reference tree was available at build time)
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libgprm_ref.so")

_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)
_D = C.POINTER(C.c_double)
_U8 = C.POINTER(C.c_ubyte)


def _f(a):
    return a.ctypes.data_as(_F)


def _i(a):
    return a.ctypes.data_as(_I)


def soa(q: np.ndarray) -> np.ndarray:
    """(n, ndof) -> contiguous SoA buffer q[i + n*j] (offset = n)."""
    return np.ascontiguousarray(np.asarray(q, np.float32).T).reshape(-1)


def _load_oracle():
    if not os.path.exists(ORACLE_LIB):
        raise RuntimeError(f"{ORACLE_LIB} missing: run `make -C oracle`")
    lib = C.CDLL(ORACLE_LIB)
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.c_void_p]
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_check_configs.argtypes = [C.c_void_p, _F, C.c_int, C.c_int, C.c_int, C.c_float, _I, _F, _U8]
    lib.orc_check_edges.argtypes = [C.c_void_p, _F, _F, C.c_int, C.c_int, C.c_float, C.c_int,
                                    C.c_float, _I, C.POINTER(C.c_int64)]
    lib.orc_edge_steps.argtypes = [C.c_void_p, _F, _F, C.c_int, C.c_int, C.c_float, C.c_int, _I, _F]
    lib.orc_edge_testnum.argtypes = [_F, _F, C.c_int, C.c_int, C.c_int, C.c_float, _I]
    lib.orc_count_ops_configs.argtypes = [C.c_void_p, _F, C.c_int, C.c_int, _D]
    lib.orc_count_ops_edges.argtypes = [C.c_void_p, _F, _F, C.c_int, C.c_int, C.c_float, _D]
    lib.orc_forward_kinematics.argtypes = [C.c_void_p, _F, C.c_int, _F]
    lib.orc_sincos64.argtypes = [_D, C.c_int, _D, _D]
    lib.orc_edge_classify.argtypes = [C.c_void_p, _F, _F, C.c_int, C.c_int, C.c_float, C.c_int, C.c_float,
                                      _U8, _I, _I]
    lib.orc_config_classify.argtypes = [C.c_void_p, _F, C.c_int, C.c_int, C.c_int, C.c_float, _U8, _I]
    lib.orc_band_pair_range.argtypes = [C.c_void_p, _F, C.c_int, C.c_int, C.c_int, C.c_float, _I, _I, _I]
    lib.orc_check_configs64_range.argtypes = [C.c_void_p, _F, C.c_int, C.c_int, _I, _I, _I]
    return lib


# mode bits of the oracle's checks
FP32, FP64, FP32_BAND, DEVICE_TRIG = 0, 1, 2, 4

OP_NAMES = ["add", "mul", "div", "sqrt", "trig", "cmp", "pairs", "iters", "climb_dots", "checks"]


class Oracle:
    """The restated algorithm on one scene."""

    def __init__(self, scene):
        from gpuprm_b200._abi import DescHolder
        self.lib = _load_oracle()
        self.scene = scene
        self._desc = DescHolder(scene)
        self.h = self.lib.orc_create(C.addressof(self._desc.desc))
        if not self.h:
            raise ValueError("oracle rejected the scene")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def check_configs(self, q: np.ndarray, mode: int = 0, band: float = 1e-5):
        """q: (n, ndof). Returns (codes int32, margins float32, inband bool)."""
        n = q.shape[0]
        buf = soa(q)
        code = np.zeros(n, np.int32)
        margin = np.zeros(n, np.float32)
        ib = np.zeros(n, np.uint8)
        self.lib.orc_check_configs(self.h, _f(buf), n, n, mode, band, _i(code), _f(margin),
                                   ib.ctypes.data_as(_U8))
        return code, margin, ib.astype(bool)

    def band_pair_range(self, q: np.ndarray, mode: int = DEVICE_TRIG, band: float = 1e-5):
        """The pairs [lo, hi) an FP64 recheck of each configuration has to
        test, from its FP32 pair loop (first pair decided within the band;
        one past the last such pair when free, the pair count when
        colliding), and the FP32 codes."""
        n = q.shape[0]
        buf = soa(q)
        lo, hi, code = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
        self.lib.orc_band_pair_range(self.h, _f(buf), n, n, mode, band, _i(lo), _i(hi), _i(code))
        return lo, hi, code

    def check_configs64_range(self, q: np.ndarray, lo: np.ndarray, hi: np.ndarray):
        """FP64 codes of the configurations over their pairs [lo, hi)."""
        n = q.shape[0]
        buf = soa(q)
        lo = np.ascontiguousarray(lo, np.int32)
        hi = np.ascontiguousarray(hi, np.int32)
        code = np.zeros(n, np.int32)
        self.lib.orc_check_configs64_range(self.h, _f(buf), n, n, _i(lo), _i(hi), _i(code))
        return code

    def check_edges(self, qs: np.ndarray, qe: np.ndarray, dq: float, mode: int = 0,
                    band: float = 1e-5):
        """Returns (res int32 = code of last colliding step, total steps)."""
        n = qs.shape[0]
        bs, be = soa(qs), soa(qe)
        res = np.zeros(n, np.int32)
        steps = C.c_int64(0)
        self.lib.orc_check_edges(self.h, _f(bs), _f(be), n, n, dq, mode, band, _i(res),
                                 C.byref(steps))
        return res, int(steps.value)

    def edge_classify(self, qs: np.ndarray, qe: np.ndarray, dq: float, mode: int = DEVICE_TRIG,
                      band: float = 1e-5, threads: int = 1):
        """Verdict classes of edges (orc_edge_classify): returns (cls uint8:
        0 free outside the band, 1 colliding outside the band, 2 decided in
        the band; band_res int32, the FP32 + FP64-band result; inband_steps
        int32).  threads > 1 splits the edges over host threads (the scene
        is read-only and ctypes releases the GIL during the call)."""
        n = qs.shape[0]
        cls = np.zeros(n, np.uint8)
        res = np.zeros(n, np.int32)
        nin = np.zeros(n, np.int32)

        def run(lo, hi):
            m = hi - lo
            if m <= 0:
                return
            bs, be = soa(qs[lo:hi]), soa(qe[lo:hi])
            c, r, k = np.zeros(m, np.uint8), np.zeros(m, np.int32), np.zeros(m, np.int32)
            self.lib.orc_edge_classify(self.h, _f(bs), _f(be), m, m, dq, mode, band, c.ctypes.data_as(_U8),
                                       _i(r), _i(k))
            cls[lo:hi], res[lo:hi], nin[lo:hi] = c, r, k

        _split(run, n, threads)
        return cls, res, nin

    def config_classify(self, q: np.ndarray, mode: int = DEVICE_TRIG, band: float = 1e-5, threads: int = 1):
        """Verdict classes of vertex checks (orc_config_classify): returns
        (cls uint8 as in edge_classify, band_code int32)."""
        n = q.shape[0]
        cls = np.zeros(n, np.uint8)
        code = np.zeros(n, np.int32)

        def run(lo, hi):
            m = hi - lo
            if m <= 0:
                return
            buf = soa(q[lo:hi])
            c, k = np.zeros(m, np.uint8), np.zeros(m, np.int32)
            self.lib.orc_config_classify(self.h, _f(buf), m, m, mode, band, c.ctypes.data_as(_U8), _i(k))
            cls[lo:hi], code[lo:hi] = c, k

        _split(run, n, threads)
        return cls, code

    def edge_steps(self, qs, qe, dq, mode: int = 0):
        n = qs.shape[0]
        tn = self.testnum(qs, qe, dq)
        tot = int(tn.sum())
        codes = np.zeros(tot, np.int32)
        margins = np.zeros(tot, np.float32)
        bs, be = soa(qs), soa(qe)
        self.lib.orc_edge_steps(self.h, _f(bs), _f(be), n, n, dq, mode, _i(codes), _f(margins))
        return tn, codes, margins

    def testnum(self, qs, qe, dq):
        n = qs.shape[0]
        bs, be = soa(qs), soa(qe)
        tn = np.zeros(n, np.int32)
        self.lib.orc_edge_testnum(_f(bs), _f(be), n, n, self.scene.ndof, dq, _i(tn))
        return tn

    def count_ops_configs(self, q):
        n = q.shape[0]
        buf = soa(q)
        out = np.zeros(10, np.float64)
        self.lib.orc_count_ops_configs(self.h, _f(buf), n, n, out.ctypes.data_as(_D))
        return dict(zip(OP_NAMES, out.tolist()))

    def count_ops_edges(self, qs, qe, dq):
        n = qs.shape[0]
        bs, be = soa(qs), soa(qe)
        out = np.zeros(10, np.float64)
        self.lib.orc_count_ops_edges(self.h, _f(bs), _f(be), n, n, dq, out.ctypes.data_as(_D))
        return dict(zip(OP_NAMES, out.tolist()))

    def forward_kinematics(self, q, mode: int = 0):
        out = np.zeros((self.scene.ndof + 1) * 12, np.float32)
        qq = np.ascontiguousarray(np.asarray(q, np.float32))
        self.lib.orc_forward_kinematics(self.h, _f(qq), mode, _f(out))
        return out.reshape(self.scene.ndof + 1, 4, 3)


def _split(fn, n: int, threads: int, chunk: int = 64):
    """Runs fn(lo, hi) over [0, n) in pieces of `chunk` items on `threads`
    host threads (work-stealing order; each piece is independent)."""
    threads = max(1, int(threads))
    if threads == 1 or n <= chunk:
        fn(0, n)
        return
    import threading
    lock = threading.Lock()
    nxt = [0]
    err = []

    def worker():
        while True:
            with lock:
                lo = nxt[0]
                nxt[0] += chunk
            if lo >= n or err:
                return
            try:
                fn(lo, min(n, lo + chunk))
            except Exception as e:   # surfaced after join
                err.append(e)
                return

    ts = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if err:
        raise err[0]


def sincos64(x: np.ndarray):
    lib = _load_oracle()
    x = np.ascontiguousarray(np.asarray(x, np.float64))
    s = np.zeros_like(x)
    c = np.zeros_like(x)
    lib.orc_sincos64(x.ctypes.data_as(_D), x.size, s.ctypes.data_as(_D), c.ctypes.data_as(_D))
    return s, c


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _load_ref():
    lib = C.CDLL(REF_LIB)
    lib.ref_open.restype = C.c_void_p
    lib.ref_open.argtypes = [C.c_char_p, C.c_int, C.c_float, C.c_int]
    lib.ref_close.argtypes = [C.c_void_p]
    lib.ref_indicator.argtypes = [C.c_void_p, _F]
    lib.ref_check_configs.argtypes = [C.c_void_p, _F, C.c_int, C.c_int, _I]
    lib.ref_check_edges.argtypes = [C.c_void_p, _F, _F, C.c_int, C.c_int, _I]
    lib.ref_check_edges_mt.argtypes = [C.c_char_p, C.c_int, C.c_float, C.c_int, _F, _F, C.c_int,
                                       C.c_int, _I, C.c_int, C.c_int]
    lib.ref_check_configs_mt.argtypes = [C.c_char_p, C.c_int, _F, C.c_int, C.c_int, _I, C.c_int,
                                         C.c_int]
    return lib


class RefChecker:
    """The reference's RobotConfigspace<ndof> CPU path on a scene written to a
    config directory."""

    def __init__(self, scene, dq: float = 0.01, nbuf: int = 4096, config_dir: str = None):
        from gpuprm_b200.scenes import write_config_dir
        if not ref_available():
            raise RuntimeError(f"{REF_LIB} missing")
        self.lib = _load_ref()
        self.scene = scene
        self.dq = dq
        self.nbuf = nbuf
        if config_dir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="gprm_scene_")
            config_dir = self._tmp.name
            write_config_dir(scene, config_dir)
        self.dir = config_dir
        self.h = self.lib.ref_open(config_dir.encode(), scene.ndof, dq, nbuf)
        if not self.h:
            raise RuntimeError("reference failed to open the scene")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_close(self.h)
            self.h = None

    def check_configs(self, q):
        n = q.shape[0]
        buf = soa(q)
        code = np.zeros(n, np.int32)
        self.lib.ref_check_configs(self.h, _f(buf), n, n, _i(code))
        return code

    def check_edges(self, qs, qe):
        n = qs.shape[0]
        bs, be = soa(qs), soa(qe)
        res = np.zeros(n, np.int32)
        self.lib.ref_check_edges(self.h, _f(bs), _f(be), n, n, _i(res))
        return res

    def check_edges_mt(self, qs, qe, nthreads, chunk=64):
        n = qs.shape[0]
        bs, be = soa(qs), soa(qe)
        res = np.zeros(n, np.int32)
        self.lib.ref_check_edges_mt(self.dir.encode(), self.scene.ndof, self.dq, self.nbuf,
                                    _f(bs), _f(be), n, n, _i(res), nthreads, chunk)
        return res

    def check_configs_mt(self, q, nthreads, chunk=256):
        n = q.shape[0]
        buf = soa(q)
        code = np.zeros(n, np.int32)
        self.lib.ref_check_configs_mt(self.dir.encode(), self.scene.ndof, _f(buf), n, n,
                                      _i(code), nthreads, chunk)
        return code
