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
