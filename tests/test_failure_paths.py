"""Failure paths, made on the host or by bounded device waits (B200).

* FP64 queue overflow: a test hook caps the recheck queue far below the
  checks that need it; the overflow pass must complete the results on the
  stream, on the host-buffer, device-pointer and batched entry points alike
  (vertex codes and the edge codes of both policies identical: the early
  exit's code is that of the first colliding step in the check kernel's
  order, overflowed or not), and count the recomputed items.
* Device allocation failure: a test hook fails the n-th device allocation;
  the call returns GPRM_ERR_NOMEM and the handle works on the next call.
* Tensor-core waits: a test hook shrinks the clock budget of the MLP
  kernels' pipeline waits until they expire; the kernel drains its own
  copies and MMAs and returns, the device status reports it, and after the
  budget is restored the same calls give the same bits as before.
No test faults, traps or hangs the GPU: every wait involved is bounded and
every failure is made on the host or by such a budget.
"""
import numpy as np
import pytest

from conftest import load_golden
from gpuprm_b200 import scenes
from gpuprm_b200._abi import (GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT, GPRM_MODE_FAST,
                              GPRM_MODE_FP64_BAND)
from gpuprm_b200.configspace import GprmError, RobotConfigspace

pytestmark = pytest.mark.gpu

MODES = {"exact": GPRM_MODE_FP64_BAND, "fast": GPRM_MODE_FP64_BAND | GPRM_MODE_FAST}
GPRM_ERR_NOMEM = -5


def _dev(a):
    import torch
    return torch.tensor(np.ascontiguousarray(np.asarray(a, np.float32).T), device="cuda:0")


def _device_edges(cs, qs, qe):
    import torch
    res = torch.zeros(len(qs), dtype=torch.int32, device="cuda:0")
    cs.check_edges_device(_dev(qs), _dev(qe), res)
    torch.cuda.synchronize()
    return res.cpu().numpy()


def _device_configs(cs, q):
    import torch
    res = torch.zeros(len(q), dtype=torch.int32, device="cuda:0")
    cs.check_configs_device(_dev(q), res)
    torch.cuda.synchronize()
    return res.cpu().numpy()


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_queue_overflow_gives_complete_results(arith):
    sc, z = load_golden("box4")
    dq = float(z["dq"])
    qs, qe, q = z["qs"], z["qe"], z["q"]
    cs = RobotConfigspace(sc, dq=dq)
    cs.init()
    cs.set_mode(MODES[arith])
    want = {}
    for pol in (GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT):
        cs.set_edge_policy(pol)
        want[pol] = cs.check_edges(qs, qe)
    want_cfg = cs.check_configs(q)
    st0 = cs.stats()
    assert st0["band_rechecks"] > 40 and st0["band_overflow_items"] == 0
    cs.lib.gprm_debug_set_queue_capacity(cs.h, 4)
    try:
        for pol in (GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT):
            cs.set_edge_policy(pol)
            for got in (cs.check_edges(qs, qe), _device_edges(cs, qs, qe)):
                np.testing.assert_array_equal(got, want[pol])
        np.testing.assert_array_equal(cs.check_configs(q), want_cfg)
        np.testing.assert_array_equal(_device_configs(cs, q), want_cfg)
    finally:
        cs.lib.gprm_debug_set_queue_capacity(cs.h, 0)
    st1 = cs.stats()
    assert st1["band_overflow_items"] > 0
    # and the uncapped queue again: nothing overflows
    cs.set_edge_policy(GPRM_EDGES_ALL_STEPS)
    np.testing.assert_array_equal(cs.check_edges(qs, qe), want[GPRM_EDGES_ALL_STEPS])
    assert cs.stats()["band_overflow_items"] == st1["band_overflow_items"]


@pytest.mark.parametrize("pol", [GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT])
def test_batched_queue_overflow_gives_complete_results(pol):
    import torch
    from gpuprm_b200.batch import CONFIGS, EDGES, ProblemBatch, pack_items
    scs = [scenes.make_box4(41), scenes.make_hull6(42), scenes.make_box4(43)]
    spaces = []
    for sc in scs:
        cs = RobotConfigspace(sc, dq=0.02)
        cs.init()
        cs.set_mode(GPRM_MODE_FP64_BAND)
        cs.set_edge_policy(pol)
        spaces.append(cs)
    qv = [scenes.uniform_configs(sc, 700, 50 + i) for i, sc in enumerate(scs)]
    ed = [scenes.random_edges(sc, 150, 60 + i, 0.6) for i, sc in enumerate(scs)]
    Q, ov = pack_items(qv)
    A, oe = pack_items([e[0] for e in ed])
    B_, _ = pack_items([e[1] for e in ed])
    Q, A, B_ = (torch.tensor(x, device="cuda:0") for x in (Q, A, B_))
    out = {}
    for cap in (0, 4):
        b = ProblemBatch(spaces)
        b.set_layout(CONFIGS, ov, queue_capacity=cap)
        b.set_layout(EDGES, oe, queue_capacity=cap)
        rv = torch.zeros(Q.shape[1], dtype=torch.int32, device="cuda:0")
        re = torch.zeros(A.shape[1], dtype=torch.int32, device="cuda:0")
        b.check_configs_device(Q, rv)
        b.check_edges_device(A, B_, re)
        torch.cuda.synchronize()
        out[cap] = (rv.cpu().numpy(), re.cpu().numpy(), b.stats())
    np.testing.assert_array_equal(out[4][0], out[0][0])
    np.testing.assert_array_equal(out[4][1], out[0][1])
    assert out[0][2]["band_overflow_items"] == 0 and out[4][2]["band_overflow_items"] > 0
    assert out[4][2]["band_rechecks"] > 8


def test_device_alloc_failure_returns_nomem_and_the_handle_recovers():
    sc, z = load_golden("hull6")
    dq = float(z["dq"])
    qs, qe = z["qs"], z["qe"]
    cs = RobotConfigspace(sc, dq=dq)
    cs.init()
    cs.set_mode(GPRM_MODE_FP64_BAND)
    cs.set_edge_policy(GPRM_EDGES_ALL_STEPS)
    want = cs.check_edges(qs, qe)
    lib = cs.lib
    # each larger batch grows the request's buffers: fail the 1st, then the
    # 3rd allocation of that growth (some buffers already replaced)
    for reps, nth in ((4, 1), (8, 3)):
        a, b = np.tile(qs, (reps, 1)), np.tile(qe, (reps, 1))
        lib.gprm_debug_fail_device_alloc(nth)
        with pytest.raises(GprmError) as e:
            cs.check_edges(a, b)
        assert e.value.status == GPRM_ERR_NOMEM
        lib.gprm_debug_fail_device_alloc(0)
        np.testing.assert_array_equal(cs.check_edges(a, b), np.tile(want, reps))
    # the device-pointer entry point's scratch, the same way
    a, b = np.tile(qs, (16, 1)), np.tile(qe, (16, 1))
    lib.gprm_debug_fail_device_alloc(2)
    with pytest.raises(GprmError) as e:
        _device_edges(cs, a, b)
    assert e.value.status == GPRM_ERR_NOMEM
    lib.gprm_debug_fail_device_alloc(0)
    np.testing.assert_array_equal(_device_edges(cs, a, b), np.tile(want, 16))


def test_mlp_wait_budget_expiry_is_reported_and_recovers():
    import torch
    from gpuprm_b200.mlp import CollisionMLP
    rng = np.random.default_rng(7)
    q = torch.tensor(rng.uniform(-np.pi, np.pi, (6, 8192)).astype(np.float32), device="cuda:0")
    y = torch.tensor((rng.random(8192) < 0.4).astype(np.float32), device="cuda:0")
    mlp = CollisionMLP(6, seed=3)
    want = mlp.predict(q).clone()
    g0, l0 = mlp.gradients(q, y)
    assert mlp.device_status() == 0
    # fused inference: waits of 64 cycles cannot see their copies or MMAs
    mlp.set_wait_budget(64)
    mlp.predict(q)
    assert mlp.device_status() != 0
    mlp.set_wait_budget(0)
    assert mlp.device_status() == 0
    assert torch.equal(mlp.predict(q), want)
    # the training GEMMs the same way
    mlp.set_wait_budget(64)
    mlp.gradients(q, y)
    assert mlp.device_status() != 0
    mlp.set_wait_budget(0)
    g1, l1 = mlp.gradients(q, y)
    assert mlp.device_status() == 0
    np.testing.assert_array_equal(g1, g0)          # gradients reduce in a fixed order
    assert abs(l1 - l0) <= 1e-5 * abs(l0)           # the reported loss is summed atomically


def test_queue_grows_to_the_demand_of_a_dense_band_scene():
    """A cluttered scene where most edge steps end in the FP64 band (96% of
    its configurations collide, most of them in shallow contact): the first
    device-pointer call overflows the default queue and completes through
    the overflow pass; the handle reads that demand back without a
    synchronisation and sizes the next call's queue to it, so the same call
    again overflows nothing and gives the same codes (both policies)."""
    import torch
    from gpuprm_b200.workloads import knn_pairs
    sc = scenes.make_mixed(141)
    q = torch.tensor(np.ascontiguousarray(scenes.uniform_configs(sc, 1 << 16, 7).T), device="cuda:0")
    for pol in (GPRM_EDGES_EARLY_EXIT, GPRM_EDGES_ALL_STEPS):
        cs = RobotConfigspace(sc, dq=0.01)
        cs.init()
        cs.set_mode(GPRM_MODE_FP64_BAND | GPRM_MODE_FAST)
        cs.set_edge_policy(pol)
        codes = torch.zeros(q.shape[1], dtype=torch.int32, device="cuda:0")
        cs.check_configs_device(q, codes)
        qf = q[:, codes == 0].T.contiguous()
        i, j = knn_pairs(qf, 10)
        qs, qe = qf[i].T.contiguous(), qf[j].T.contiguous()
        n = qs.shape[1]
        assert n > 10000
        outs, ovf = [], []
        for _ in range(3):
            res = torch.zeros(n, dtype=torch.int32, device="cuda:0")
            before = cs.stats()["band_overflow_items"]
            cs.check_edges_device(qs, qe, res)
            torch.cuda.synchronize()
            ovf.append(cs.stats()["band_overflow_items"] - before)
            outs.append(res.cpu().numpy())
        assert ovf[0] > 0 and ovf[1] == 0 and ovf[2] == 0
        np.testing.assert_array_equal(outs[1], outs[0])
        np.testing.assert_array_equal(outs[2], outs[0])
