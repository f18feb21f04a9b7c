"""GPUPRM's own planner with the B200 checker dropped in.

oracle/_ref/prm_dropin compiles the reference's PRMSolver (prmsolver.cpp,
unmodified, single-rank MPI stand-in) and runs it on the reference scene
with either checker behind Configspace<4>.  The reference run's stored
roadmap (store_results, prmsolver.cpp:2947-3055) is pinned in
tests/golden/prm_dropin_config1.json by make_prm_golden.py.  With the B200
checker in FP32 mode the planner must draw the same random numbers and
store byte-identical results: every verdict it asked for was the same.
"""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_prm_golden as G  # noqa: E402

FIX = json.load(open(G.FIXTURE))
needs_bin = pytest.mark.skipif(not os.path.exists(G.BIN), reason="oracle/_ref/prm_dropin not built")


def test_fixture_is_complete():
    assert FIX["counters"]["num_nodes"] > 0
    assert FIX["files"]["connection.bin"] == "01"          # the planner connected start and goal
    for g in ("graphl", "graphr"):
        for f in ("qstorage.bin", "edgesfrom.bin", "edgesto.bin", "edgesweight.bin", "path.bin", "pathc.bin"):
            assert f"{g}/{f}" in FIX["files"]


@needs_bin
@pytest.mark.skipif(not os.path.isdir("/root/reference/prm"), reason="reference tree absent")
def test_reference_run_reproduces_fixture_and_writer_matches_store_results(tmp_path):
    """The reference run still gives the fixture, and gpuprm_b200.results,
    fed the planner's final roadmaps (raw arrays dumped by the harness),
    writes the same 33 files byte for byte as the planner's own
    store_results (prmsolver.cpp:2947-3055)."""
    from gpuprm_b200 import results as R
    dump = str(tmp_path / "dump")
    line, files = G.run_planner("ref", str(tmp_path), ["--dump", dump])
    assert files == FIX["files"]
    for k, v in FIX["counters"].items():
        assert line[k] == v, k
    connected = open(os.path.join(dump, "connection.bin"), "rb").read()[0] == 1
    mine = str(tmp_path / "mine")
    R.store_results(mine, R.load_dump(os.path.join(dump, "graphl")), R.load_dump(os.path.join(dump, "graphr")),
                    connected)
    assert G.digest_outputs(mine) == FIX["files"]


@needs_bin
@pytest.mark.gpu
def test_b200_checker_builds_the_same_roadmap(tmp_path):
    line, files = G.run_planner("b200", str(tmp_path), ["--mode", "fp32"])
    print("reference checker plan s:", FIX["reference_plan_seconds"], " B200 checker plan s:", line["plan_seconds"])
    for k, v in FIX["counters"].items():
        assert line[k] == v, k
    assert files == FIX["files"]
