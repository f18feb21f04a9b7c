"""Parity of the CUDA checker with the oracle and the reference (B200).

Every call goes through the C ABI (libgprm_b200.so).  The bars:
  * FP32 mode: codes bit-identical to the oracle's F32D arithmetic (the
    reference's operations with correctly rounded joint trigonometry);
    free/colliding verdicts identical to the reference's golden verdicts.
  * FP64 band mode: codes bit-identical to the oracle's FP32+FP64-band result.
  * edges: ALL_STEPS codes bit-identical to the oracle (last colliding step,
    like the reference CPU path); EARLY_EXIT verdicts identical.
"""
import numpy as np
import pytest

from conftest import GOLDEN_NAMES, load_golden
from gpuprm_b200 import scenes
from gpuprm_b200._abi import (GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT, GPRM_MODE_FP32,
                              GPRM_MODE_FP64_BAND)
from gpuprm_b200.configspace import GprmError, RobotConfigspace
import oracle as O

pytestmark = pytest.mark.gpu


def space(sc, dq, mode=GPRM_MODE_FP32, policy=GPRM_EDGES_ALL_STEPS, nbuf=0):
    cs = RobotConfigspace(sc, dq=dq, nbuf=nbuf)
    cs.init()
    cs.set_mode(mode)
    cs.set_edge_policy(policy)
    return cs


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_forward_kinematics_bitexact(name):
    sc, z = load_golden(name)
    cs = space(sc, float(z["dq"]))
    orc = O.Oracle(sc)
    for q in z["q"][:64]:
        np.testing.assert_array_equal(cs.debug_fk(q), orc.forward_kinematics(q, O.DEVICE_TRIG))


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_vertex_fp32_bitexact(name):
    sc, z = load_golden(name)
    cs = space(sc, float(z["dq"]))
    got = cs.check_configs(z["q"])
    want, _, _ = O.Oracle(sc).check_configs(z["q"], O.FP32 | O.DEVICE_TRIG)
    np.testing.assert_array_equal(got, want)
    # verdicts equal the reference's own CPU checker
    np.testing.assert_array_equal(got != 0, z["codes"] != 0)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_vertex_band_bitexact(name):
    sc, z = load_golden(name)
    cs = space(sc, float(z["dq"]), mode=GPRM_MODE_FP64_BAND)
    got = cs.check_configs(z["q"])
    want, _, ib = O.Oracle(sc).check_configs(z["q"], O.FP32_BAND | O.DEVICE_TRIG)
    np.testing.assert_array_equal(got, want)
    st = cs.stats()
    assert st["band_rechecks"] == int(ib.sum())


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_edges_all_steps_bitexact(name):
    sc, z = load_golden(name)
    dq = float(z["dq"])
    cs = space(sc, dq)
    got = cs.check_edges(z["qs"], z["qe"])
    want, steps = O.Oracle(sc).check_edges(z["qs"], z["qe"], dq, O.FP32 | O.DEVICE_TRIG)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(got != 0, z["edge_res"] != 0)
    st = cs.stats()
    assert st["edge_steps_nominal"] == steps


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_edges_band_all_steps_bitexact(name):
    sc, z = load_golden(name)
    dq = float(z["dq"])
    cs = space(sc, dq, mode=GPRM_MODE_FP64_BAND)
    got = cs.check_edges(z["qs"], z["qe"])
    want, _ = O.Oracle(sc).check_edges(z["qs"], z["qe"], dq, O.FP32_BAND | O.DEVICE_TRIG)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("mode", [GPRM_MODE_FP32, GPRM_MODE_FP64_BAND])
@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_edges_early_exit_verdicts(name, mode):
    sc, z = load_golden(name)
    dq = float(z["dq"])
    cs = space(sc, dq, mode=mode, policy=GPRM_EDGES_EARLY_EXIT)
    got = cs.check_edges(z["qs"], z["qe"])
    omode = (O.FP32 if mode == GPRM_MODE_FP32 else O.FP32_BAND) | O.DEVICE_TRIG
    want, steps = O.Oracle(sc).check_edges(z["qs"], z["qe"], dq, omode)
    np.testing.assert_array_equal(got != 0, want != 0)
    st = cs.stats()
    assert st["edge_steps_nominal"] == steps
    assert st["edge_steps_executed"] <= steps
    # deterministic: same codes on a second run
    np.testing.assert_array_equal(cs.check_edges(z["qs"], z["qe"]), got)


def test_generated_scenes_larger_sample():
    for sc, dq, n, ne in ((scenes.make_hull6(31), 0.01, 20000, 1500),
                          (scenes.make_wall7(32, num_obstacles=160), 0.01, 6000, 400)):
        orc = O.Oracle(sc)
        cs = space(sc, dq, mode=GPRM_MODE_FP64_BAND)
        q = scenes.uniform_configs(sc, n, 5)
        np.testing.assert_array_equal(cs.check_configs(q), orc.check_configs(q, O.FP32_BAND | O.DEVICE_TRIG)[0])
        qs, qe = scenes.random_edges(sc, ne, 6, 0.6)
        want, _ = orc.check_edges(qs, qe, dq, O.FP32_BAND | O.DEVICE_TRIG)
        cs.set_edge_policy(GPRM_EDGES_ALL_STEPS)
        np.testing.assert_array_equal(cs.check_edges(qs, qe), want)
        cs.set_edge_policy(GPRM_EDGES_EARLY_EXIT)
        np.testing.assert_array_equal(cs.check_edges(qs, qe) != 0, want != 0)


@pytest.mark.parametrize("mode", [GPRM_MODE_FP32, GPRM_MODE_FP64_BAND])
@pytest.mark.parametrize("policy", [GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT])
def test_split_edges_match_whole_edges(policy, mode):
    """Batches of at most 16384 edges split long edges over several warps
    (segments of seg_rounds x 32 steps, at most 64 per edge): codes and
    nominal step counts equal those of one warp per edge, and the all-steps
    codes equal the oracle's."""
    sc = scenes.make_hull6(5)
    dq = 0.003
    qs, qe = scenes.random_edges(sc, 300, 11, 9.0)           # up to ~3000 steps (> 64 rounds)
    cs = space(sc, dq, mode=mode, policy=policy)
    out = {}
    for split in ((0, 4), (16384, 4), (16384, 2), (16384, 1)):
        cs.set_edge_split(*split)
        s0 = cs.stats()["edge_steps_nominal"]
        out[split] = (cs.check_edges(qs, qe), cs.stats()["edge_steps_nominal"] - s0)
    whole, steps = out[(0, 4)]
    assert steps > 64 * 32 * 10
    assert (whole != 0).any() and (whole == 0).any()
    for split, (codes, n) in out.items():
        np.testing.assert_array_equal(codes, whole, err_msg=str(split))
        assert n == steps
    if policy == GPRM_EDGES_ALL_STEPS:
        omode = (O.FP32 if mode == GPRM_MODE_FP32 else O.FP32_BAND) | O.DEVICE_TRIG
        want, _ = O.Oracle(sc).check_edges(qs[:48], qe[:48], dq, omode)
        np.testing.assert_array_equal(out[(16384, 1)][0][:48], want)


@pytest.mark.parametrize("policy", [GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT])
def test_split_mid_size_batches_match_whole_edges(policy):
    """Above 16384 edges the segment offsets come from the three-pass scan
    (EDGE_SEG_BLOCKS blocks): 40000 edges of up to ~1000 steps, split into
    segments of 1 or 2 rounds, give the codes and nominal step counts of
    one warp per edge."""
    sc = scenes.make_hull6(6)
    dq = 0.005
    qs, qe = scenes.random_edges(sc, 40000, 12, 5.0)
    cs = space(sc, dq, mode=GPRM_MODE_FP64_BAND, policy=policy)
    out = {}
    for split in ((0, 2), (1 << 22, 2), (1 << 22, 1), (40000, 2)):
        cs.set_edge_split(*split)
        s0 = cs.stats()
        out[split] = (cs.check_edges(qs, qe), cs.stats()["edge_steps_nominal"] - s0["edge_steps_nominal"],
                      cs.stats()["launches"] - s0["launches"])
    whole, steps, launches = out[(0, 2)]
    assert (whole != 0).any() and (whole == 0).any()
    for split, (codes, n, nl) in out.items():
        np.testing.assert_array_equal(codes, whole, err_msg=str(split))
        assert n == steps
        if split[0] >= 40000:
            assert nl == launches + 3          # the three scan passes


def test_edge_split_arguments():
    sc = scenes.make_box4(1)
    cs = space(sc, 0.02)
    for bad in ((-1, 4), ((1 << 22) + 1, 4), (100, 0)):
        with pytest.raises(GprmError):
            cs.set_edge_split(*bad)
    cs.set_edge_split(0, 4)


def test_edge_cases():
    sc = scenes.make_box4(8)
    cs = space(sc, 0.02, mode=GPRM_MODE_FP64_BAND)
    # empty batches
    assert cs.check_configs(np.zeros((0, 4), np.float32)).shape == (0,)
    assert cs.check_edges(np.zeros((0, 4), np.float32), np.zeros((0, 4), np.float32)).shape == (0,)
    # out of bounds -> 1 (check_boundaries first, robotconfigspace.cpp:315)
    q = np.array([[0, 0, 0, 4.0], [0, 0, 0, 0]], np.float32)
    codes = cs.check_configs(q)
    assert codes[0] == 1
    # single-config indicator equals the batched one
    assert cs.indicator(q[1]) == codes[1]
    # NaN configuration: cap (-1), like the reference
    assert cs.check_configs(np.full((1, 4), np.nan, np.float32))[0] in (-1, 1)
    # testnum = 1 edge -> -1 (0/0 lerp, robotconfigspace.cpp:411-413)
    qs = np.full((1, 4), 0.2, np.float32)
    qe = qs + np.float32(0.001)
    assert cs.check_edges(qs, qe)[0] == -1
    # infinite edge -> error, not a fault
    bad = qs.copy()
    bad[0, 0] = np.inf
    with pytest.raises(GprmError):
        cs.check_edges(qs, bad)
    # the handle stays usable after the error
    assert cs.check_configs(q)[0] == 1


def test_async_requests_out_of_order():
    sc, z = load_golden("box4")
    dq = float(z["dq"])
    cs = space(sc, dq, policy=GPRM_EDGES_ALL_STEPS, nbuf=512)
    want, _ = O.Oracle(sc).check_edges(z["qs"], z["qe"], dq, O.FP32 | O.DEVICE_TRIG)
    n = len(want)
    parts = [slice(0, n // 3), slice(n // 3, 2 * n // 3), slice(2 * n // 3, n)]
    bufs = []
    for s in parts:
        qs = np.ascontiguousarray(z["qs"][s].T).reshape(-1)
        qe = np.ascontiguousarray(z["qe"][s].T).reshape(-1)
        res = np.zeros(s.stop - s.start, np.int32)
        m = s.stop - s.start
        bufs.append((res, cs.indicator2_async(qs, qe, res, m, m)))
    for res, req in reversed(bufs):
        cs.indicator2_async_wait(req)
    np.testing.assert_array_equal(np.concatenate([b[0] for b in bufs]), want)
    with pytest.raises(GprmError):
        cs.indicator2_async_wait(12345)
    # N > nbuf is refused like the reference's assert (robotconfigspace.cpp:618)
    with pytest.raises(GprmError):
        big = np.zeros((600, 4), np.float32)
        cs.check_edges(big, big)


def test_device_pointer_api_matches_host_api():
    import torch
    sc, z = load_golden("hull6")
    dq = float(z["dq"])
    cs = space(sc, dq, mode=GPRM_MODE_FP64_BAND, policy=GPRM_EDGES_ALL_STEPS)
    host_res = cs.check_edges(z["qs"], z["qe"])
    host_codes = cs.check_configs(z["q"])
    dev = torch.device("cuda:0")
    qs = torch.tensor(np.ascontiguousarray(z["qs"].T), device=dev)
    qe = torch.tensor(np.ascontiguousarray(z["qe"].T), device=dev)
    res = torch.zeros(len(host_res), dtype=torch.int32, device=dev)
    cs.check_edges_device(qs, qe, res)
    q = torch.tensor(np.ascontiguousarray(z["q"].T), device=dev)
    codes = torch.zeros(len(host_codes), dtype=torch.int32, device=dev)
    cs.check_configs_device(q, codes)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(res.cpu().numpy(), host_res)
    np.testing.assert_array_equal(codes.cpu().numpy(), host_codes)


@pytest.mark.parametrize("policy", [GPRM_EDGES_EARLY_EXIT, GPRM_EDGES_ALL_STEPS])
def test_host_api_in_parts_matches_device_api(policy):
    """Host-buffer requests of 2^16 items or more run in parts (staging and
    transfer of one part under the checks of the previous one); results equal
    the device-pointer entry point's, for edges and configurations, with an
    item count that does not divide evenly."""
    import torch
    from gpuprm_b200 import scenes
    sc = scenes.make_hull6(5)
    cs = space(sc, 0.01, mode=GPRM_MODE_FP64_BAND, policy=policy)
    qs, qe = scenes.random_edges(sc, 70001, 6, 0.6)
    q = scenes.uniform_configs(sc, 100003, 7)
    host_e = cs.check_edges(qs, qe)
    host_v = cs.check_configs(q)
    dev = torch.device("cuda:0")
    tqs = torch.tensor(np.ascontiguousarray(qs.T), device=dev)
    tqe = torch.tensor(np.ascontiguousarray(qe.T), device=dev)
    res = torch.zeros(len(host_e), dtype=torch.int32, device=dev)
    cs.check_edges_device(tqs, tqe, res)
    tq = torch.tensor(np.ascontiguousarray(q.T), device=dev)
    codes = torch.zeros(len(host_v), dtype=torch.int32, device=dev)
    cs.check_configs_device(tq, codes)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(res.cpu().numpy(), host_e)
    np.testing.assert_array_equal(codes.cpu().numpy(), host_v)
    assert (host_e != 0).any() and (host_e == 0).any()


@pytest.mark.parametrize("band", [0.0, 1e-3, 2e-2])
def test_band_width_changes_nothing_but_the_band(band):
    """The separation certificates depend on the band; results must equal
    the oracle's for every band width."""
    sc, z = load_golden("hull6")
    dq = float(z["dq"])
    cs = space(sc, dq, mode=GPRM_MODE_FP64_BAND)
    cs.set_band(band)
    orc = O.Oracle(sc)
    want, _, _ = orc.check_configs(z["q"], O.FP32_BAND | O.DEVICE_TRIG, band=band)
    np.testing.assert_array_equal(cs.check_configs(z["q"]), want)
    want_e, _ = orc.check_edges(z["qs"], z["qe"], dq, O.FP32_BAND | O.DEVICE_TRIG, band=band)
    np.testing.assert_array_equal(cs.check_edges(z["qs"], z["qe"]), want_e)


def test_certificates_settle_most_pairs():
    sc, z = load_golden("hull6")
    cs = space(sc, float(z["dq"]))
    cs.check_configs(z["q"])
    st = cs.stats()
    assert st["pairs_certified"] > 4 * st["pairs_tested"]


def test_handles_keep_their_launch_shapes():
    """Launch shapes are per handle: configuring a second handle with a
    smaller shared-memory footprint must not break the first one."""
    sc, z = load_golden("hull6")
    a = space(sc, float(z["dq"]), mode=GPRM_MODE_FP64_BAND)
    want = a.check_configs(z["q"])
    a.set_launch(True, 128, True)
    assert a.get_launch(True)["scene_in_smem"]
    b = space(scenes.make_box4(3), 0.02, mode=GPRM_MODE_FP64_BAND)
    b.check_configs(scenes.uniform_configs(scenes.make_box4(3), 100, 1))
    np.testing.assert_array_equal(a.check_configs(z["q"]), want)


@pytest.mark.gpu
def test_compressed_edge_check_equals_the_expanded_pairs():
    """indicator2(qs, M, qe, res, posqe, numqe, offset), the star-shaped
    form the reference declares but leaves unimplemented in its robot space:
    res[l] is the code of the edge qs[k] -> qe[l] for l in k's range (the
    array space's meaning), later ranges overwrite earlier ones, uncovered
    entries keep their value, and bad ranges are rejected."""
    from gpuprm_b200.configspace import GprmError
    sc, z = load_golden("hull6")
    cs = RobotConfigspace(sc, dq=float(z["dq"]))
    cs.init()
    rng = np.random.default_rng(5)
    M, L = 40, 300
    qs = scenes.uniform_configs(sc, M, 11)
    qe = scenes.uniform_configs(sc, L, 12)
    qe = qe * 0.3 + np.repeat(qs, (L + M - 1) // M, axis=0)[:L] * 0.7     # ends near the starts
    pos = rng.integers(0, L - 20, M).astype(np.int32)
    num = rng.integers(0, 20, M).astype(np.int32)
    num[3] = 0
    res = np.full(L, -77, np.int32)
    cs.indicator2_compressed(np.ascontiguousarray(qs.T), M, np.ascontiguousarray(qe.T), res, pos, num, L)
    want = np.full(L, -77, np.int32)
    for k in range(M):
        ls = np.arange(pos[k], pos[k] + num[k])
        if len(ls):
            want[ls] = cs.check_edges(np.repeat(qs[k:k + 1], len(ls), axis=0), qe[ls])
    np.testing.assert_array_equal(res, want)
    assert (res != -77).sum() > 100 and (res == -77).any()
    bad = num.copy()
    bad[0] = L
    with pytest.raises(GprmError):
        cs.indicator2_compressed(np.ascontiguousarray(qs.T), M, np.ascontiguousarray(qe.T), res, pos, bad, L)
