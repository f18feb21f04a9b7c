"""Batched near-node sampler: the Philox restatement pinned by the published
known-answer vectors, the kernel equal to it bit for bit, and the batched
sampler equal to a one-candidate-at-a-time restatement of get_random_nodes
(prmsolver.cpp:2585-2624) with the oracle's vertex check."""
import numpy as np
import pytest

import sampler_oracle as SO


def test_philox_known_answer_vectors():
    """Philox4x32-10 vectors published with the Random123 library."""
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for c, k, want in kat:
        got = SO.philox4x32_10(*[np.array([x]) for x in c], *k)
        assert tuple(int(g[0]) for g in got) == want


def test_acceptance_follows_surrnum():
    rng = np.random.default_rng(0)
    nodes = rng.uniform(-1, 1, (2, 3)).astype(np.float32)
    for s, p in ((0, 3), (1, 3), (3, 2)):
        _, par = SO.candidates(nodes, [s, s], p, 0.1, 5, 0, 20000)
        rate = (par >= 0).mean()
        assert abs(rate - 1.0 / (1 + s) ** p) < 0.02


@pytest.mark.gpu
@pytest.mark.parametrize("ndof,power,D", [(4, 3, 1.0), (7, 2, 0.3)])
def test_gpu_candidates_match_oracle(ndof, power, D):
    import torch
    from gpuprm_b200.sampler import candidates
    rng = np.random.default_rng(1)
    nodes = rng.uniform(-3, 3, (5000, ndof)).astype(np.float32)
    surr = rng.integers(0, 6, 5000).astype(np.int32)
    dev = torch.device("cuda:0")
    q, par = candidates(torch.tensor(np.ascontiguousarray(nodes.T), device=dev), torch.tensor(surr, device=dev),
                        D, seed=0x123456789, t0=(1 << 33) + 7, B=30000, power=power)
    wq, wp = SO.candidates(nodes, surr, power, D, 0x123456789, (1 << 33) + 7, 30000)
    np.testing.assert_array_equal(par.cpu().numpy(), wp)
    np.testing.assert_array_equal(q.cpu().numpy().T, wq)


@pytest.mark.gpu
def test_gpu_sample_near_matches_sequential_restatement():
    import torch
    from conftest import load_golden
    from gpuprm_b200.configspace import RobotConfigspace
    from gpuprm_b200.sampler import sample_near
    from gpuprm_b200._abi import GPRM_MODE_FP64_BAND
    import oracle as O
    sc, z = load_golden("box4")
    cs = RobotConfigspace(sc, dq=0.02)
    cs.init()
    cs.set_mode(GPRM_MODE_FP64_BAND)
    orc = O.Oracle(sc)
    nodes = z["q"][cs.check_configs(z["q"]) == 0][:300].astype(np.float32)
    surr = np.random.default_rng(2).integers(0, 4, len(nodes)).astype(np.int32)
    dev = torch.device("cuda:0")
    q, par, used = sample_near(cs, torch.tensor(np.ascontiguousarray(nodes.T), device=dev),
                               torch.tensor(surr, device=dev), num=500, D=0.5, seed=42, batch=1024)
    free = lambda qq: orc.check_configs(qq, O.FP32_BAND | O.DEVICE_TRIG)[0] == 0
    wq, wp, wused = SO.sample_near(nodes, surr, 3, 0.5, 42, 500, free, batch=4096)
    assert used == wused
    np.testing.assert_array_equal(par.cpu().numpy(), wp)
    np.testing.assert_array_equal(q.cpu().numpy().T, wq)


@pytest.mark.gpu
def test_gpu_block_candidates_match_oracle():
    """The block-storage draw (gprm_sample_near_blocks) equals the
    restatement bit for bit, with an empty block and a block reaching past
    the node slots among the blocks passed (both dismiss)."""
    import torch
    from gpuprm_b200.sampler import candidates
    rng = np.random.default_rng(4)
    n = 3000
    nodes = rng.uniform(-3, 3, (n, 6)).astype(np.float32)
    surr = rng.integers(0, 5, n).astype(np.int32)
    pos = np.array([0, 256, 512, 900, 1300, 2000, 2990, 2995], np.int32)
    num = np.array([256, 3, 100, 0, 256, 1, 5, 40], np.int32)     # the last runs past n
    dev = torch.device("cuda:0")
    T = lambda a: torch.tensor(a, device=dev)
    q, par = candidates(T(np.ascontiguousarray(nodes.T)), T(surr), 0.4, seed=99, t0=5, B=50000, power=3,
                        blocks=(T(pos), T(num)))
    wq, wp = SO.candidates(nodes, surr, 3, 0.4, 99, 5, 50000, pos, num)
    np.testing.assert_array_equal(par.cpu().numpy(), wp)
    np.testing.assert_array_equal(q.cpu().numpy().T, wq)
    p = par.cpu().numpy()
    assert (p >= 0).any() and not np.isin(p, np.arange(900, 1300)).any()
