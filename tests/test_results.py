"""Roadmap output in the reference's store_results format: a device
planner's roadmap written with gpuprm_b200.results reads back consistently
(the byte-for-byte comparison with the reference's own writer is in
tests/test_dropin.py)."""
import numpy as np
import pytest

from gpuprm_b200 import results as R


def test_from_edges_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    q = rng.uniform(-3, 3, (600, 4)).astype(np.float32)
    ei = rng.integers(0, 600, 1500)
    ej = rng.integers(0, 600, 1500)
    keep = ei != ej
    ei, ej = ei[keep], ej[keep]
    path = [5, int(ej[ei == 5][0]) if (ei == 5).any() else 6]
    g = R.Roadmap.from_edges(q, ei, ej, start=path[0], end=path[-1], path=path)
    R.store_results(str(tmp_path / "out"), g, R.Roadmap.from_edges(q[:1], [], [], 0, 0), True)
    d = R.load_graph(str(tmp_path / "out" / "graphl"), 4)
    assert d["numc"][0] == 600 and d["newblockpos"][0] == 768 and d["blocknum"][0] == 3
    np.testing.assert_array_equal(d["qstoragec"], q)
    assert len(d["edgesfrom"]) == 2 * len(ei)           # both directions, like the reference
    np.testing.assert_array_equal(np.sort(d["surrnum"][:600]), np.sort(np.bincount(np.concatenate([ei, ej]), minlength=600)))
    np.testing.assert_array_equal(d["path"], np.array(path[::-1], np.int32))   # goal first
    assert d["startc"][0] == path[0] and d["endc"][0] == path[-1]
    assert open(tmp_path / "out" / "connection.bin", "rb").read()[0] == 1


@pytest.mark.gpu
def test_device_planner_roadmap_in_reference_format(tmp_path):
    import torch
    from gpuprm_b200 import planner, scenes
    from gpuprm_b200.configspace import RobotConfigspace
    sc = scenes.make_box4(3)
    cs = RobotConfigspace(sc, dq=0.02)
    cs.init()
    starts, goals = planner.make_queries(cs, sc, 20, seed=1)
    r = planner.plain_prm(cs, sc, starts, goals, 1 << 13, k=10, seed=2, keep_roadmap=True)
    t = int(np.argmax(r.success))
    assert r.success[t]
    verts, ei, ej = r.info["roadmap"]
    R.store_plan(str(tmp_path / "plan"), r, verts, ei, ej, query=t)
    d = R.load_graph(str(tmp_path / "plan" / "graphl"), sc.ndof)
    n = verts.shape[0]
    assert d["numc"][0] == n + 2
    path = d["path"][::-1]                                  # start first
    assert path[0] == n and path[-1] == n + 1
    np.testing.assert_array_equal(d["qstoragec"][path], r.paths[t])
    edges = set(zip(d["edgesfrom"].tolist(), d["edgesto"].tolist()))
    assert all((int(a), int(b)) in edges for a, b in zip(path[:-1], path[1:]))
