"""Verdict parity with the reference CPU checker by band class (B200).

The north-star bar: every check whose FP32 separation margin lies outside
the FP64 band gets the reference's free / not-free verdict; every check
inside the band gets the FP64 oracle's.  The oracle classifies each
configuration or edge (oracle/parity.py, orc_edge_classify) and the
reference's own CPU checker (oracle/_ref, compiled from its sources) gives
the verdicts to match.  Both arithmetic variants are held to it: the exact
FP32 path (whose codes are also bit-identical to the oracle, see
test_gpu_parity.py) and the fast path (GPRM_MODE_FAST: contracted
arithmetic, table-started support climbs), whose codes may differ by
rounding.

Sizes: the golden fixtures (reference codes recorded by
tests/golden/make_golden.py); 20,000 kNN edges of the headline hull6 roadmap
construction (the benchmark's edge distribution); a sample of the full
512-obstacle 7-DOF wall scene of the stress configuration.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN_NAMES, load_golden
from gpuprm_b200 import scenes
from gpuprm_b200._abi import (GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT, GPRM_MODE_FAST,
                              GPRM_MODE_FP64_BAND)
from gpuprm_b200.configspace import RobotConfigspace
import oracle as O
import parity as P

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
MODES = {"exact": GPRM_MODE_FP64_BAND, "fast": GPRM_MODE_FP64_BAND | GPRM_MODE_FAST}
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/libgprm_ref.so not built")


def space(sc, dq, arith, policy=GPRM_EDGES_EARLY_EXIT):
    cs = RobotConfigspace(sc, dq=dq)
    cs.init()
    cs.set_mode(MODES[arith])
    cs.set_edge_policy(policy)
    return cs


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_golden_verdicts_by_band_class(name, arith):
    sc, z = load_golden(name)
    dq = float(z["dq"])
    orc = O.Oracle(sc)
    cs = space(sc, dq, arith)
    got = cs.check_configs(z["q"])
    np.testing.assert_array_equal(cs.check_configs(z["q"]), got)          # deterministic
    cls, band = orc.config_classify(z["q"], threads=THREADS)
    d = P.verdict_parity(got, z["codes"], cls, band)
    assert P.parity_ok(d), d
    cls, band, nin = orc.edge_classify(z["qs"], z["qe"], dq, threads=THREADS)
    for policy in (GPRM_EDGES_EARLY_EXIT, GPRM_EDGES_ALL_STEPS):
        cs.set_edge_policy(policy)
        got_e = cs.check_edges(z["qs"], z["qe"])
        d = P.verdict_parity(got_e, z["edge_res"], cls, band, nin)
        assert P.parity_ok(d), (policy, d)


def _knn_edges(kind, seed, n_samples, k, m, device="cuda:0"):
    """m seeded edges of the kNN roadmap of n_samples uniform samples (the
    benchmark's construction), as (m, ndof) host arrays."""
    import torch
    from gpuprm_b200 import workloads
    ws = workloads.edge_workload(kind, seed=seed, n_samples=n_samples, k=k, device=device)
    E = ws["qs"].shape[1]
    pick = np.random.default_rng(seed + 1).permutation(E)[:m]
    qs = np.ascontiguousarray(ws["qs"].T.cpu().numpy()[pick])
    qe = np.ascontiguousarray(ws["qe"].T.cpu().numpy()[pick])
    del ws
    torch.cuda.synchronize()
    return qs, qe


@needs_ref
def test_hull6_knn_edges_vs_reference():
    """20,000 edges of the hull6 kNN roadmap (k = 10, dq = 0.01), early
    exit, FP64 band: zero verdict mismatches with the reference outside the
    band, zero with the FP64 oracle inside it, in both arithmetic variants."""
    dq = 0.01
    sc = scenes.make_scene("hull6", 0)
    qs, qe = _knn_edges("hull6", 0, 1 << 16, 10, 20000)
    ref = O.RefChecker(sc, dq=dq, nbuf=4096).check_edges_mt(qs, qe, THREADS, chunk=16)
    cls, band, nin = O.Oracle(sc).edge_classify(qs, qe, dq, threads=THREADS)
    assert (cls == 0).sum() > 5000 and (cls == 1).sum() > 1000      # both verdicts well represented
    for arith in ("exact", "fast"):
        cs = space(sc, dq, arith)
        got = cs.check_edges(qs, qe)
        d = P.verdict_parity(got, ref, cls, band, nin)
        assert P.parity_ok(d), (arith, d)


def test_wall7_full_scene_vs_oracle():
    """The stress configuration's full scene (7 DOF, 512 obstacles, 4117
    pairs): 4096 uniform configurations and 512 kNN edges of free samples
    (k = 16, dq = 0.005) against the oracle's classes, and against the
    reference where it is built."""
    dq = 0.005
    sc = scenes.make_scene("wall7", 0)
    assert len(sc.pair_from) > 4000
    orc = O.Oracle(sc)
    q = scenes.uniform_configs(sc, 4096, 21)
    ccls, cband = orc.config_classify(q, threads=THREADS)
    qs, qe = _knn_edges("wall7", 0, 1 << 15, 16, 512)
    ecls, eband, nin = orc.edge_classify(qs, qe, dq, threads=THREADS)
    cref = eref = None
    if O.ref_available():
        ref = O.RefChecker(sc, dq=dq, nbuf=4096)
        cref = ref.check_configs_mt(q, THREADS, chunk=64)
        eref = ref.check_edges_mt(qs, qe, THREADS, chunk=4)
    for arith in ("exact", "fast"):
        cs = space(sc, dq, arith)
        got = cs.check_configs(q)
        d = P.verdict_parity(got, cref if cref is not None else cband, ccls, cband)
        assert P.parity_ok(d), (arith, "configs", d)
        got_e = cs.check_edges(qs, qe)
        d = P.verdict_parity(got_e, eref if eref is not None else eband, ecls, eband, nin)
        assert P.parity_ok(d), (arith, "edges", d)
