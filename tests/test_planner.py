"""Roadmap planners: plain vs lazy vs learned (B200)."""
import numpy as np
import pytest

from gpuprm_b200 import planner


@pytest.mark.gpu
def test_lazy_prm_has_the_connectivity_of_the_eager_prm():
    """Lazy checking (Boruvka rounds, lazy query attachment) solves exactly
    the queries the eager PRM solves on the same samples, checking fewer
    edges; every path verifies.  So do the two-round schedule and a single
    round that checks every candidate edge."""
    from gpuprm_b200 import scenes
    from gpuprm_b200._abi import GPRM_MODE_FP64_BAND
    from gpuprm_b200.configspace import RobotConfigspace
    sc = scenes.make_hull6(0)
    cs = RobotConfigspace(sc, dq=0.01)
    cs.init()
    cs.set_mode(GPRM_MODE_FP64_BAND)
    starts, goals = planner.make_queries(cs, sc, 200, seed=3)
    plain = planner.plain_prm(cs, sc, starts, goals, 1 << 14, k=10, seed=4)
    lazy = planner.lazy_prm(cs, sc, starts, goals, 1 << 14, k=10, seed=4)
    np.testing.assert_array_equal(plain.success, lazy.success)
    assert plain.info["verified"] and lazy.info["verified"]
    assert lazy.edge_checks < plain.edge_checks
    assert plain.success.mean() > 0.2
    for kw in (dict(max_rounds=2, first=2), dict(max_rounds=1), dict(max_rounds=8, first=1, growth=1)):
        other = planner.lazy_prm(cs, sc, starts, goals, 1 << 14, k=10, seed=4, **kw)
        np.testing.assert_array_equal(plain.success, other.success)
        assert other.info["verified"]


@pytest.mark.gpu
def test_learned_guidance_prunes_and_keeps_paths_verified():
    from gpuprm_b200 import scenes
    from gpuprm_b200._abi import GPRM_MODE_FP64_BAND
    from gpuprm_b200.configspace import RobotConfigspace
    sc = scenes.make_hull6(0)
    cs = RobotConfigspace(sc, dq=0.01)
    cs.init()
    cs.set_mode(GPRM_MODE_FP64_BAND)
    mlp, losses, _, _ = planner.train_predictor(cs, sc, n_labels=1 << 17, epochs=3)
    starts, goals = planner.make_queries(cs, sc, 200, seed=5)
    plain = planner.plain_prm(cs, sc, starts, goals, 1 << 14, k=10, seed=6)
    learned = planner.lazy_prm(cs, sc, starts, goals, 1 << 14, k=10, seed=6, mlp=mlp)
    lazy = planner.lazy_prm(cs, sc, starts, goals, 1 << 14, k=10, seed=6)
    assert learned.info["verified"]
    assert learned.info["pruned"] > 0
    assert learned.edge_steps < plain.edge_steps
    # what the network adds to the same lazy planner on the same samples:
    # fewer vertex checks (pruning) and fewer cross-component checks (ordering)
    assert learned.vertex_checks < lazy.vertex_checks
    assert learned.info["later_edges"] < lazy.info["later_edges"]
    # every reported path connects its own start and goal
    for i, p in enumerate(learned.paths):
        if p is not None:
            assert np.array_equal(p[0], starts[i]) and np.array_equal(p[-1], goals[i])


@pytest.mark.gpu
def test_radius_roadmap_matches_a_brute_force_pair_list():
    """With a C-space radius the candidate edges are every pair of free
    vertices closer than it (the reference's connection rule on the 4-DOF
    box scene); the eager and lazy PRMs answer the same pairs on them and
    every path verifies."""
    import torch
    from gpuprm_b200 import scenes
    from gpuprm_b200._abi import GPRM_MODE_FP64_BAND
    from gpuprm_b200.configspace import RobotConfigspace
    from gpuprm_b200.neighbours import NeighbourIndex
    sc = scenes.make_box4(0)
    cs = RobotConfigspace(sc, dq=0.02)
    cs.init()
    cs.set_mode(GPRM_MODE_FP64_BAND)
    rng = np.random.default_rng(9)
    verts = torch.tensor(rng.uniform(-np.pi, np.pi, (3000, 4)).astype(np.float32), device="cuda:0")
    i, j = planner._index_and_pairs(NeighbourIndex(4), verts, 10, radius=1.0, cap=256)
    v = verts.cpu().numpy().astype(np.float64)
    d = np.linalg.norm(v[:, None, :] - v[None, :, :], axis=2)
    got = set(zip(i.cpu().numpy().tolist(), j.cpu().numpy().tolist()))
    # float32 distances within 1e-5 of the radius may round either way
    inner = set(zip(*(x.tolist() for x in np.nonzero(np.triu(d < 1.0 - 1e-5, 1)))))
    outer = set(zip(*(x.tolist() for x in np.nonzero(np.triu(d < 1.0 + 1e-5, 1)))))
    assert len(inner) > 1000
    assert inner <= got <= outer
    starts, goals = planner.make_queries(cs, sc, 20, seed=3)
    plain = planner.plain_prm(cs, sc, starts, goals, 1 << 16, seed=4, radius=0.5)
    lazy = planner.lazy_prm(cs, sc, starts, goals, 1 << 16, seed=4, radius=0.5)
    np.testing.assert_array_equal(plain.success, lazy.success)
    assert plain.info["verified"] and lazy.info["verified"]
    assert plain.success.mean() > 0.8
