"""Many problems per launch: batched results equal each problem's own
results bit for bit (and the oracle's), graph replay equals the direct
call, the autotuner keeps a shape that fits, bad layouts are rejected."""
import numpy as np
import pytest

from gpuprm_b200 import scenes
from gpuprm_b200._abi import GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT, GPRM_MODE_FP32, GPRM_MODE_FP64_BAND
from gpuprm_b200.batch import CONFIGS, EDGES, offsets_of, pack_items
import oracle as O


def test_pack_items_layout():
    a = np.arange(6, dtype=np.float32).reshape(3, 2)
    b = np.arange(100, 108, dtype=np.float32).reshape(2, 4)
    out, offs = pack_items([a, b], rows=5)
    assert offs.tolist() == [0, 3, 5]
    assert out.shape == (5, 5)
    np.testing.assert_array_equal(out[:2, :3], a.T)
    np.testing.assert_array_equal(out[:4, 3:], b.T)
    assert not out[2:, :3].any() and not out[4:, 3:].any()
    assert offsets_of([]).tolist() == [0]


def _problems(count, mode, policy, seed=0):
    from gpuprm_b200.configspace import RobotConfigspace
    rng = np.random.default_rng(seed)
    out = []
    for p in range(count):
        sc = scenes.make_mixed(1000 + seed * 100 + p)
        dq = float(rng.choice([0.01, 0.02, 0.03]))
        cs = RobotConfigspace(sc, dq=dq)
        cs.init()
        cs.set_mode(mode)
        cs.set_edge_policy(policy)
        out.append((sc, dq, cs))
    return out


def _inputs(probs, seed, nq_range=(0, 700), ne_range=(0, 300)):
    rng = np.random.default_rng(seed)
    qs_all, qa_all, qb_all = [], [], []
    for p, (sc, dq, cs) in enumerate(probs):
        nq = int(rng.integers(*nq_range))
        ne = int(rng.integers(*ne_range))
        qs_all.append(scenes.uniform_configs(sc, nq, seed * 37 + p))
        a, b = scenes.random_edges(sc, ne, seed * 41 + p, 0.5)
        qa_all.append(a)
        qb_all.append(b)
    return qs_all, qa_all, qb_all


@pytest.mark.gpu
@pytest.mark.parametrize("mode,policy", [(GPRM_MODE_FP64_BAND, GPRM_EDGES_ALL_STEPS),
                                         (GPRM_MODE_FP64_BAND, GPRM_EDGES_EARLY_EXIT),
                                         (GPRM_MODE_FP32, GPRM_EDGES_ALL_STEPS)])
def test_batch_equals_per_problem(mode, policy):
    import torch
    from gpuprm_b200.batch import ProblemBatch
    probs = _problems(12, mode, policy, seed=1)
    qv, qa, qb = _inputs(probs, 3)
    qv[2] = qv[2][:0]            # an empty problem in the middle
    want_v = [cs.check_configs(q) if len(q) else np.zeros(0, np.int32) for (sc, dq, cs), q in zip(probs, qv)]
    want_e = [cs.check_edges(a, b) if len(a) else np.zeros(0, np.int32) for (sc, dq, cs), a, b in zip(probs, qa, qb)]
    B = ProblemBatch([cs for _, _, cs in probs])
    Q, offs_v = pack_items(qv)
    A, offs_e = pack_items(qa)
    Bq, _ = pack_items(qb)
    dev = torch.device("cuda:0")
    Qd, Ad, Bd = (torch.tensor(x, device=dev) for x in (Q, A, Bq))
    rv = torch.full((Q.shape[1],), -7, dtype=torch.int32, device=dev)
    re = torch.full((A.shape[1],), -7, dtype=torch.int32, device=dev)
    B.set_layout(CONFIGS, offs_v)
    B.set_layout(EDGES, offs_e)
    B.check_configs_device(Qd, rv)
    B.check_edges_device(Ad, Bd, re)
    torch.cuda.synchronize()
    got_v, got_e = rv.cpu().numpy(), re.cpu().numpy()
    for p in range(len(probs)):
        np.testing.assert_array_equal(got_v[offs_v[p]:offs_v[p + 1]], want_v[p], err_msg=f"configs {p}")
        if policy == GPRM_EDGES_ALL_STEPS:
            np.testing.assert_array_equal(got_e[offs_e[p]:offs_e[p + 1]], want_e[p], err_msg=f"edges {p}")
        else:
            np.testing.assert_array_equal(got_e[offs_e[p]:offs_e[p + 1]] != 0, want_e[p] != 0, err_msg=f"edges {p}")
    st = B.stats()
    assert st["vertex_checks"] == Q.shape[1]
    assert st["edge_steps_nominal"] > 0


@pytest.mark.gpu
def test_batch_matches_oracle():
    import torch
    from gpuprm_b200.batch import ProblemBatch
    probs = _problems(3, GPRM_MODE_FP64_BAND, GPRM_EDGES_ALL_STEPS, seed=2)
    qv, qa, qb = _inputs(probs, 5, (200, 400), (60, 120))
    B = ProblemBatch([cs for _, _, cs in probs])
    Q, offs_v = pack_items(qv)
    A, offs_e = pack_items(qa)
    Bq, _ = pack_items(qb)
    dev = torch.device("cuda:0")
    Qd, Ad, Bd = (torch.tensor(x, device=dev) for x in (Q, A, Bq))
    rv = torch.zeros(Q.shape[1], dtype=torch.int32, device=dev)
    re = torch.zeros(A.shape[1], dtype=torch.int32, device=dev)
    B.set_layout(CONFIGS, offs_v)
    B.set_layout(EDGES, offs_e)
    B.check_configs_device(Qd, rv)
    B.check_edges_device(Ad, Bd, re)
    torch.cuda.synchronize()
    for p, (sc, dq, cs) in enumerate(probs):
        orc = O.Oracle(sc)
        want, _, _ = orc.check_configs(qv[p], O.FP32_BAND | O.DEVICE_TRIG)
        np.testing.assert_array_equal(rv.cpu().numpy()[offs_v[p]:offs_v[p + 1]], want)
        want_e, _ = orc.check_edges(qa[p], qb[p], dq, O.FP32_BAND | O.DEVICE_TRIG)
        np.testing.assert_array_equal(re.cpu().numpy()[offs_e[p]:offs_e[p + 1]], want_e)


@pytest.mark.gpu
def test_graph_replay_and_autotune():
    import torch
    from gpuprm_b200.batch import ProblemBatch
    probs = _problems(6, GPRM_MODE_FP64_BAND, GPRM_EDGES_EARLY_EXIT, seed=3)
    qv, qa, qb = _inputs(probs, 7, (100, 2000), (50, 400))
    B = ProblemBatch([cs for _, _, cs in probs])
    Q, offs_v = pack_items(qv)
    A, offs_e = pack_items(qa)
    Bq, _ = pack_items(qb)
    dev = torch.device("cuda:0")
    Qd, Ad, Bd = (torch.tensor(x, device=dev) for x in (Q, A, Bq))
    B.set_layout(CONFIGS, offs_v)
    B.set_layout(EDGES, offs_e)
    r1 = torch.zeros(Q.shape[1], dtype=torch.int32, device=dev)
    e1 = torch.zeros(A.shape[1], dtype=torch.int32, device=dev)
    B.check_configs_device(Qd, r1)
    B.check_edges_device(Ad, Bd, e1)
    tv = B.autotune(CONFIGS, Qd, None, torch.zeros_like(r1), reps=1)
    te = B.autotune(EDGES, Ad, Bd, torch.zeros_like(e1), reps=1)
    assert tv["threads"] in (64, 128, 256, 512) and tv["ms"] > 0
    assert B.get_launch(EDGES)["threads"] == te["threads"]
    assert B.get_launch(EDGES)["blocks_per_sm"] == te["blocks_per_sm"] >= 1
    table = B.tune_table(EDGES)
    assert len(table) >= 4 and min(r["ms"] for r in table) == pytest.approx(te["ms"])
    assert {r["threads"] for r in table} >= {64, 128, 256}
    assert {r["solo_min_items"] for r in table} >= {-1, 0}
    # problems in their own launches give the same results: all of them,
    # the larger ones, none
    for min_items in (0, 300, -1):
        for kind in (CONFIGS, EDGES):
            B.set_solo_threshold(kind, min_items)
        st = B.get_solo_threshold(EDGES)
        assert st["min_items"] == min_items
        assert (st["solo_problems"] == 0) == (min_items < 0)
        r4 = torch.full_like(r1, -9)
        e4 = torch.full_like(e1, -9)
        B.check_configs_device(Qd, r4)
        B.check_edges_device(Ad, Bd, e4)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(r4.cpu().numpy(), r1.cpu().numpy())
        np.testing.assert_array_equal(e4.cpu().numpy(), e1.cpu().numpy())
    for kind in (CONFIGS, EDGES):
        B.set_solo_threshold(kind, 300)
    # a capped shape (2 resident blocks per SM, the carveout as a launch
    # attribute) gives the same results, directly and in a captured graph
    for kind in (CONFIGS, EDGES):
        B.set_launch(kind, 128, 2)
        sh = B.get_launch(kind)
        assert sh["blocks_per_sm"] == 2 and sh["warps_per_sm"] == 8
    r3 = torch.full_like(r1, -9)
    e3 = torch.full_like(e1, -9)
    B.check_configs_device(Qd, r3)
    B.check_edges_device(Ad, Bd, e3)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(r3.cpu().numpy(), r1.cpu().numpy())
    np.testing.assert_array_equal(e3.cpu().numpy(), e1.cpu().numpy())
    r2 = torch.full_like(r1, -9)
    e2 = torch.full_like(e1, -9)
    B.capture(CONFIGS, Qd, None, r2)
    B.capture(EDGES, Ad, Bd, e2)
    before = B.stats()
    for _ in range(2):
        B.replay(CONFIGS)
        B.replay(EDGES)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(r2.cpu().numpy(), r1.cpu().numpy())
    np.testing.assert_array_equal(e2.cpu().numpy(), e1.cpu().numpy())
    after = B.stats()
    assert after["vertex_checks"] == before["vertex_checks"] + 2 * Q.shape[1]
    assert 5 * after["edge_steps_nominal"] == 7 * before["edge_steps_nominal"]   # 5 calls, then 2 replays


@pytest.mark.gpu
def test_batch_rejects_bad_input():
    import torch
    from gpuprm_b200.batch import ProblemBatch
    from gpuprm_b200.configspace import GprmError
    probs = _problems(2, GPRM_MODE_FP64_BAND, GPRM_EDGES_ALL_STEPS, seed=4)
    B = ProblemBatch([cs for _, _, cs in probs])
    with pytest.raises(GprmError):
        B.set_layout(CONFIGS, [1, 2, 3])          # must start at 0
    with pytest.raises(GprmError):
        B.set_layout(CONFIGS, [0, 5, 3])          # decreasing
    q = torch.zeros((7, 4), device="cuda:0")
    r = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    with pytest.raises(GprmError):
        B.check_configs_device(q, r)              # no layout yet
    B.set_layout(CONFIGS, [0, 3, 6])
    with pytest.raises(GprmError):
        B.check_configs_device(q, r)              # stride 4 < 6 items
    with pytest.raises(GprmError):
        B.replay(CONFIGS)                         # nothing captured
    probs[1][2].set_band(1e-3)
    with pytest.raises(GprmError):
        ProblemBatch([cs for _, _, cs in probs])  # bands differ
