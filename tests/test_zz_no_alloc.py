"""The no-allocation vertex-check entry point (B200).

gprm_indicator_batch_device_noalloc serves callers that may not allocate
device memory while they run (real-time planning loops, hosts whose device
memory belongs to another allocator): its work buffers are a fixed array
inside the library.  It must return exactly what the allocating entry
point gprm_indicator_batch_device returns, on consecutive calls that reuse
the shared array.  This file is collected last so that a failure here comes
after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from gpuprm_b200._abi import GPRM_MODE_FP64_BAND, GPRM_NOALLOC_MAX_CONFIGS
from gpuprm_b200.configspace import RobotConfigspace

pytestmark = pytest.mark.gpu


def _soa(q):
    import torch
    return torch.tensor(np.ascontiguousarray(np.asarray(q, np.float32).T), device="cuda:0")


@pytest.mark.parametrize("name", ["hull6", "box4"])
def test_noalloc_matches_allocating_entry_point(name):
    import torch
    sc, z = load_golden(name)
    cs = RobotConfigspace(sc, dq=float(z["dq"]))
    cs.init()
    cs.set_mode(GPRM_MODE_FP64_BAND)   # exercises the FP64 recheck queue in the scratch array
    lib, h = cs.lib, cs.h
    q = _soa(z["q"])
    n = int(q.shape[1])
    stream = torch.cuda.current_stream().cuda_stream

    want = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    assert lib.gprm_indicator_batch_device(h, C.c_void_p(q.data_ptr()), C.c_void_p(want.data_ptr()), n, n,
                                           C.c_void_p(stream)) == 0
    torch.cuda.synchronize()
    rechecks = cs.stats()["band_rechecks"]   # after the allocating call
    for _ in range(2):   # two calls in a row share the same scratch array
        got = torch.full((n,), 99, dtype=torch.int32, device="cuda:0")
        rc = lib.gprm_indicator_batch_device_noalloc(h, C.c_void_p(q.data_ptr()), C.c_void_p(got.data_ptr()),
                                                     n, n, C.c_void_p(stream))
        assert rc == 0, lib.gprm_last_error(h)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy())
        # this call ran its own FP64 recheck through the queue in the shared array
        now = cs.stats()["band_rechecks"]
        assert now > rechecks
        rechecks = now


def test_noalloc_rejects_oversized_batches():
    import torch
    sc, z = load_golden("box4")
    cs = RobotConfigspace(sc, dq=float(z["dq"]))
    cs.init()
    n = GPRM_NOALLOC_MAX_CONFIGS + 1
    q = torch.zeros((sc.ndof, n), dtype=torch.float32, device="cuda:0")
    res = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    rc = cs.lib.gprm_indicator_batch_device_noalloc(cs.h, C.c_void_p(q.data_ptr()), C.c_void_p(res.data_ptr()),
                                                    n, n, None)
    assert rc == -1
    assert b"no-allocation limit" in cs.lib.gprm_last_error(cs.h)
