"""Host-side logic of the lazy planner on CPU tensors, with a fake checker:
the per-component edge selection, the exactness of the lazy rounds (the
components equal those of the fully checked graph) and the lazy query
attachment (the same (start, goal) neighbour pairs as checking every
attachment edge)."""
import numpy as np
import pytest
import torch
from scipy.sparse import coo_matrix
from scipy.sparse.csgraph import connected_components

from gpuprm_b200 import planner


def _random_graph(rng, V, E):
    a = rng.integers(0, V, 3 * E)
    b = rng.integers(0, V, 3 * E)
    keep = a != b
    key = np.unique(np.minimum(a, b)[keep] * V + np.maximum(a, b)[keep])[:E]
    rng.shuffle(key)
    return torch.tensor(key // V), torch.tensor(key % V)


def _partition(V, i, j, mask):
    m = np.asarray(mask, bool)
    g = coo_matrix((np.ones(int(m.sum())), (np.asarray(i)[m], np.asarray(j)[m])), shape=(V, V))
    _, lab = connected_components(g, directed=False)
    # canonical: the smallest vertex of each component
    first = {}
    return np.array([first.setdefault(c, v) for v, c in enumerate(lab)])


def _canon(label):
    first = {}
    return np.array([first.setdefault(int(c), v) for v, c in enumerate(np.asarray(label))])


def test_cheapest_per_component_matches_brute_force():
    rng = np.random.default_rng(0)
    for m in (1, 2, 3):
        n = 400
        rest = torch.tensor(rng.permutation(5000)[:n])
        la = torch.tensor(rng.integers(0, 40, n), dtype=torch.int32)
        lb = (la + torch.tensor(rng.integers(1, 40, n), dtype=torch.int32)) % 40
        got = set(planner._cheapest_per_component(rest, la, lb, m).tolist())
        want = set()
        for c in range(40):
            seen = [int(rest[t]) for t in range(n) if int(la[t]) == c or int(lb[t]) == c]
            want.update(seen[:m])
        assert got == want


@pytest.mark.parametrize("rounds,first,growth", [(1, 2, 2), (2, 2, 2), (4, 1, 2), (6, 1, 2), (10, 1, 1), (3, 3, 3)])
def test_lazy_rounds_give_the_components_of_the_checked_graph(rounds, first, growth):
    rng = np.random.default_rng(rounds * 100 + first * 10 + growth)
    V, E = 600, 2400
    i, j = _random_graph(rng, V, E)
    E = int(i.numel())
    free = torch.tensor(rng.random(E) < 0.55)
    cost = torch.tensor(rng.random(E), dtype=torch.float32)
    calls = []

    def check(sel):
        calls.append(sel.clone())
        return free[sel]

    good, checked, label, per_round, _ = planner._lazy_rounds(
        V, i, j, cost, check, lambda g: torch.tensor(_partition(V, i, j, g.numpy().astype(bool))),
        rounds, first, growth, planner._Phases(False), cost)
    sel = torch.cat(calls)
    assert sel.numel() == torch.unique(sel).numel()           # each edge checked at most once
    assert bool((good.bool() == (checked & free)).all())
    np.testing.assert_array_equal(_canon(label), _partition(V, i, j, free.numpy()))
    assert len(per_round) <= rounds
    if rounds > 1:
        assert int(checked.sum()) < E


def _fake_checker(w):
    def check(cs, qa, qb, policy=None):
        h = torch.frac(torch.sin(qa @ w[0] + qb @ w[1]) * 1e4)
        return (h < 0.45).to(torch.int32)                     # nonzero = colliding
    return check


def _first_pairs(ok, label, nb, Q, kk):
    """The pair choice of the planner's query attachment, given edge verdicts."""
    lab = torch.where(ok, label[nb].long(), torch.full_like(nb, -1))
    ls, lg = lab[:Q], lab[Q:]
    match = ((ls[:, :, None] == lg[:, None, :]) & (ls[:, :, None] >= 0)).reshape(Q, -1)
    has = match.any(1)
    first = torch.argmax(match.to(torch.int8), dim=1)
    return torch.where(has, first, torch.full_like(first, -1))


@pytest.mark.parametrize("seed", range(4))
def test_lazy_attachment_picks_the_pairs_of_full_checking(seed, monkeypatch):
    rng = np.random.default_rng(seed)
    d, V, Q, kk = 3, 300, 200, 6
    verts = torch.tensor(rng.random((V, d)), dtype=torch.float32)
    ends = torch.tensor(rng.random((2 * Q, d)), dtype=torch.float32)
    label = torch.tensor(rng.integers(0, 12 if seed % 2 else 40, V), dtype=torch.int32)
    nb = torch.tensor(np.stack([rng.choice(V, kk, replace=False) for _ in range(2 * Q)]))
    w = torch.tensor(rng.normal(size=(2, d)), dtype=torch.float32)
    monkeypatch.setattr(planner, "_check_edges", _fake_checker(w))
    qa = ends[:, None, :].expand(-1, kk, -1).reshape(-1, d)
    ok_all = (planner._check_edges(None, qa, verts[nb.reshape(-1)]) == 0).reshape(2 * Q, kk)
    for rounds in (0, 1, 4):
        ok, n = planner._attach_lazy(None, ends, verts, nb, label, Q, kk, rounds=rounds)
        assert bool((ok <= ok_all).all())                     # only checked edges count as free
        torch.testing.assert_close(_first_pairs(ok, label, nb, Q, kk), _first_pairs(ok_all, label, nb, Q, kk))
        assert n <= 2 * Q * kk
        if rounds:
            assert n < 2 * Q * kk


def test_lazy_rounds_without_edges():
    i = torch.zeros(0, dtype=torch.int64)
    good, checked, label, per_round, free1 = planner._lazy_rounds(
        5, i, i, torch.zeros(0), lambda sel: torch.zeros(0, dtype=torch.bool),
        lambda g: torch.arange(5, dtype=torch.int32), 4, 1, 2, planner._Phases(False))
    assert good.numel() == 0 and checked.numel() == 0 and per_round == [] and free1 == 0
    np.testing.assert_array_equal(label.numpy(), np.arange(5))


def test_cheapest_per_component_takes_whole_small_groups():
    rest = torch.tensor([7, 3, 9])
    la = torch.tensor([0, 0, 1], dtype=torch.int32)
    lb = torch.tensor([1, 2, 2], dtype=torch.int32)
    assert planner._cheapest_per_component(rest, la, lb, 10).tolist() == [3, 7, 9]
    # m = 1: component 0 -> 7, component 1 -> 7, component 2 -> 3
    assert planner._cheapest_per_component(rest, la, lb, 1).tolist() == [3, 7]


def test_lazy_attachment_skips_missing_neighbours(monkeypatch):
    """Neighbour slots marked -1 (fewer nodes than k) never count as free."""
    rng = np.random.default_rng(11)
    d, V, Q, kk = 2, 40, 30, 5
    verts = torch.tensor(rng.random((V, d)), dtype=torch.float32)
    ends = torch.tensor(rng.random((2 * Q, d)), dtype=torch.float32)
    label = torch.tensor(rng.integers(0, 3, V), dtype=torch.int32)
    nb = torch.tensor(np.stack([rng.choice(V, kk, replace=False) for _ in range(2 * Q)]))
    nb[:, -1] = -1
    w = torch.tensor(rng.normal(size=(2, d)), dtype=torch.float32)
    monkeypatch.setattr(planner, "_check_edges", _fake_checker(w))
    qa = ends[:, None, :].expand(-1, kk, -1).reshape(-1, d)
    ok_all = (planner._check_edges(None, qa, verts[nb.clamp_min(0).reshape(-1)]) == 0).reshape(2 * Q, kk)
    ok_all &= nb >= 0
    ok, n = planner._attach_lazy(None, ends, verts, nb, label, Q, kk)
    assert not bool(ok[:, -1].any())
    torch.testing.assert_close(_first_pairs(ok, label, nb.clamp_min(0), Q, kk),
                               _first_pairs(ok_all, label, nb.clamp_min(0), Q, kk))


class _FakeSpace:
    """Configurations with q[0] > 0 collide (code 4), the others are free."""

    def check_configs_device(self, q, codes):
        codes.copy_(torch.where(q[0] > 0, 4, 0).to(torch.int32))


class _FakePredictor:
    """p = a fixed function of the configuration, in [0, 1)."""

    def __init__(self, scale=1.0):
        self.scale = scale

    def predict(self, q):
        return self.scale * (0.5 + 0.5 * torch.sin(7.0 * q[1]) * torch.cos(3.0 * q[2])).clamp(0.0, 0.999)


@pytest.mark.parametrize("free_rate", [0.002, 0.01, 0.05])
def test_calibrated_prune_drops_at_most_the_free_rate(free_rate):
    """The threshold is the (1 - free_rate) quantile of p over the free
    held-out samples, clamped to [lo, hi]: at most free_rate of those
    samples lie above it (when it is not clamped)."""
    from gpuprm_b200 import scenes
    sc = scenes.make_box4(1)
    n = 1 << 14
    t = planner.calibrate_prune(_FakeSpace(), sc, _FakePredictor(), free_rate=free_rate, n=n, seed=3,
                                lo=0.0, hi=1.0, device="cpu")
    q = torch.tensor(np.ascontiguousarray(scenes.uniform_configs(sc, n, 3 + 777).T))
    p = _FakePredictor().predict(q)[q[0] <= 0]
    assert 0.0 < t < 1.0
    assert float((p > t).float().mean()) <= free_rate + 1e-3
    assert float((p >= t).float().mean()) >= free_rate - 1e-3


def test_calibrated_prune_is_clamped_and_handles_no_free_samples():
    from gpuprm_b200 import scenes
    sc = scenes.make_box4(1)
    lo = planner.calibrate_prune(_FakeSpace(), sc, _FakePredictor(scale=0.1), n=4096, device="cpu")
    assert lo == 0.9                                   # every p far below the floor
    hi = planner.calibrate_prune(_FakeSpace(), sc, _FakePredictor(scale=1.0), free_rate=1e-6, n=4096,
                                 hi=0.95, device="cpu")
    assert hi == 0.95

    class _AllColliding:
        def check_configs_device(self, q, codes):
            codes.fill_(4)
    assert planner.calibrate_prune(_AllColliding(), sc, _FakePredictor(), n=1024, device="cpu") == 0.999
