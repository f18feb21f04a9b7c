"""The CPU oracle against the reference (CPU only; no GPU).

The oracle restatement (oracle/gprm_oracle.cpp) must reproduce GPUPRM's own
CPU checker bit for bit: on the committed golden fixtures (generated by the
reference, tests/golden/make_golden.py) everywhere, and live against
oracle/_ref where the reference was compiled.
"""
import math

import numpy as np
import pytest

from conftest import GOLDEN_NAMES, load_golden
from gpuprm_b200 import scenes
import oracle as O


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_oracle_matches_reference_golden_vertices(name):
    sc, z = load_golden(name)
    codes, _, _ = O.Oracle(sc).check_configs(z["q"], O.FP32)
    np.testing.assert_array_equal(codes, z["codes"].astype(np.int32))


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_oracle_matches_reference_golden_edges(name):
    sc, z = load_golden(name)
    res, steps = O.Oracle(sc).check_edges(z["qs"], z["qe"], float(z["dq"]), O.FP32)
    np.testing.assert_array_equal(res, z["edge_res"].astype(np.int32))
    assert steps >= len(res)


@pytest.mark.skipif(not O.ref_available(), reason="reference checker not built here")
@pytest.mark.parametrize("seed", [21, 22])
def test_oracle_matches_reference_live(seed):
    for sc, dq in ((scenes.make_box4(seed), 0.02), (scenes.make_hull6(seed, num_obstacles=24), 0.01)):
        ref = O.RefChecker(sc, dq=dq, nbuf=1024)
        orc = O.Oracle(sc)
        q = scenes.uniform_configs(sc, 3000, seed)
        np.testing.assert_array_equal(orc.check_configs(q, O.FP32)[0], ref.check_configs(q))
        qs, qe = scenes.random_edges(sc, 300, seed + 1, 0.6)
        np.testing.assert_array_equal(orc.check_edges(qs, qe, dq, O.FP32)[0], ref.check_edges(qs, qe))


@pytest.mark.skipif(not O.ref_available(), reason="reference checker not built here")
def test_reference_threaded_driver_matches_serial():
    sc = scenes.make_box4(5)
    ref = O.RefChecker(sc, dq=0.02, nbuf=512)
    qs, qe = scenes.random_edges(sc, 700, 3, 0.5)
    np.testing.assert_array_equal(ref.check_edges_mt(qs, qe, 4, chunk=37), ref.check_edges(qs, qe))
    q = scenes.uniform_configs(sc, 900, 4)
    np.testing.assert_array_equal(ref.check_configs_mt(q, 3, chunk=50), ref.check_configs(q))


def _ulp_err(x, ref):
    ref = np.asarray(ref, np.float64)
    sp = np.spacing(np.abs(ref))
    return np.abs(np.asarray(x) - ref) / np.maximum(sp, np.finfo(np.float64).tiny)


def test_sincos64_error_bound():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-7, 7, 200000), rng.uniform(-1e3, 1e3, 20000),
                        np.linspace(-4 * math.pi, 4 * math.pi, 4001), [0.0, -0.0, 1e-300, 5e-324]])
    s, c = O.sincos64(x)
    assert _ulp_err(s, np.sin(x)).max() <= 4.0
    assert _ulp_err(c, np.cos(x)).max() <= 4.0
    s, c = O.sincos64(np.array([np.nan, np.inf, -np.inf]))
    assert np.all(np.isnan(s)) and np.all(np.isnan(c))


def test_sincos64_rounds_to_correct_float_nearly_always():
    """The kernels' trigonometry: sincos64 rounded to float equals the
    correctly rounded float result except where the true value sits within
    a few double ulps of a float midpoint."""
    rng = np.random.default_rng(1)
    x = rng.uniform(-math.pi, math.pi, 300000).astype(np.float32)
    s, c = O.sincos64(x.astype(np.float64))
    ref_s = np.sin(x.astype(np.float64)).astype(np.float32)
    ref_c = np.cos(x.astype(np.float64)).astype(np.float32)
    assert np.count_nonzero(s.astype(np.float32) != ref_s) <= 2
    assert np.count_nonzero(c.astype(np.float32) != ref_c) <= 2


def float_ceil(x: float) -> np.float32:
    f = np.float32(x)
    if float(f) < x:
        f = np.nextafter(f, np.float32(np.inf))
    while float(np.nextafter(f, np.float32(-np.inf))) >= x:
        f = np.nextafter(f, np.float32(-np.inf))
    return f


@pytest.mark.parametrize("thr", [-0.000001, 0.000001])
def test_float_threshold_equivalence(thr):
    """`(double)dp >= -1e-6` (collision4.h:296) equals `dp >= t` for the
    smallest float t >= -1e-6, and `(double)n < 1e-6` (collision4.h:242)
    equals `n < t'`; the kernels compare against those floats."""
    t = float_ceil(thr)
    vals = [t]
    for _ in range(40):
        vals.append(np.nextafter(vals[-1], np.float32(np.inf)))
    v = t
    for _ in range(40):
        v = np.nextafter(v, np.float32(-np.inf))
        vals.append(v)
    for f in vals:
        assert (float(f) >= thr) == bool(f >= t)
        assert (float(f) < thr) == bool(f < t)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_device_trig_changes_no_verdict(name):
    """Correctly rounded joint trigonometry (the kernels') against glibc's
    sincosf (the reference's): identical free/colliding verdicts."""
    sc, z = load_golden(name)
    orc = O.Oracle(sc)
    ref_codes = z["codes"].astype(np.int32)
    dev_codes, _, _ = orc.check_configs(z["q"], O.FP32 | O.DEVICE_TRIG)
    np.testing.assert_array_equal(dev_codes != 0, ref_codes != 0)
    assert np.mean(dev_codes != ref_codes) < 0.01
    dev_edges, _ = orc.check_edges(z["qs"], z["qe"], float(z["dq"]), O.FP32 | O.DEVICE_TRIG)
    np.testing.assert_array_equal(dev_edges != 0, z["edge_res"] != 0)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_band_mode_semantics(name):
    """FP32+band returns the FP32 code outside the band and the FP64 code
    inside it; FP32 and FP64 verdicts agree outside the band."""
    sc, z = load_golden(name)
    orc = O.Oracle(sc)
    q = z["q"]
    c32, m32, ib = orc.check_configs(q, O.FP32 | O.DEVICE_TRIG)
    c64, _, _ = orc.check_configs(q, O.FP64)
    cb, _, _ = orc.check_configs(q, O.FP32_BAND | O.DEVICE_TRIG)
    np.testing.assert_array_equal(cb[~ib], c32[~ib])
    np.testing.assert_array_equal(cb[ib], c64[ib])
    assert np.all(((c32 != 0) == (c64 != 0))[~ib])
    # every cap hit is in the band
    assert np.all(ib[c32 == -1])


def test_edge_steps_quirks():
    """testnum=1 edges (|qe-qs| < dq) evaluate c1 = 0/0 and return -1
    (robotconfigspace.cpp:411-413); step spacing is |qe-qs|/floor(|qe-qs|/dq)."""
    sc = scenes.make_box4(3)
    orc = O.Oracle(sc)
    qs = np.zeros((2, 4), np.float32) + 0.3
    qe = qs.copy()
    qe[0, 0] += 0.005   # shorter than dq
    qe[1, 1] += 0.1     # 6 steps at dq=0.02
    tn = orc.testnum(qs, qe, 0.02)
    assert list(tn) == [1, 6]
    res, steps = orc.check_edges(qs, qe, 0.02, O.FP32)
    assert res[0] == -1 and steps == 7


def test_op_counter_consistency():
    sc = scenes.make_box4(4)
    orc = O.Oracle(sc)
    q = scenes.uniform_configs(sc, 200, 9)
    ops = orc.count_ops_configs(q)
    assert ops["checks"] == 200
    assert ops["pairs"] >= ops["checks"]
    assert ops["iters"] >= ops["pairs"]
    assert ops["add"] > 0 and ops["mul"] > 0
    # counting does not change results
    codes, _, _ = orc.check_configs(q, O.FP32)
    assert codes.shape == (200,)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_band_classes_agree_with_reference(name):
    """The oracle's verdict classes (orc_config_classify, orc_edge_classify)
    against the reference's golden codes: every configuration or edge the
    oracle decides outside the band has the reference's verdict, and the
    FP32 + FP64-band results equal the existing band-mode oracle path."""
    import parity as P
    sc, z = load_golden(name)
    dq = float(z["dq"])
    orc = O.Oracle(sc)
    cls, band = orc.config_classify(z["q"], threads=4)
    d = P.verdict_parity(band, z["codes"], cls, band)
    assert d["reference_vs_class_outside_band"] == 0 and d["mismatches_outside_band"] == 0, d
    np.testing.assert_array_equal(band, orc.check_configs(z["q"], O.FP32_BAND | O.DEVICE_TRIG)[0])
    ecls, eband, nin = orc.edge_classify(z["qs"], z["qe"], dq, threads=4)
    d = P.verdict_parity(eband, z["edge_res"], ecls, eband, nin)
    assert d["reference_vs_class_outside_band"] == 0 and d["mismatches_outside_band"] == 0, d
    np.testing.assert_array_equal(eband, orc.check_edges(z["qs"], z["qe"], dq, O.FP32_BAND | O.DEVICE_TRIG)[0])
    # single-threaded and multi-threaded classification agree
    c1, b1, n1 = orc.edge_classify(z["qs"], z["qe"], dq, threads=1)
    np.testing.assert_array_equal(c1, ecls)
    np.testing.assert_array_equal(b1, eband)
    np.testing.assert_array_equal(n1, nin)
