"""The FP64 band recheck tests only a pair range (CPU, oracle).

A check the FP32 pass decides within the band is queued with the range of
pairs [lo, hi) its FP64 recheck tests: lo = the first pair decided within
the band (a collision, or a separation with margin below the band), hi =
one past the last such pair when the FP32 check is free, the pair count
when it collides.  Every pair outside the range was decided separated with
margin at least the band, so in FP64 it is separated too, and the FP64 code
over the range equals the FP64 code over every pair.  Checked here with the
oracle's own FP32 and FP64 pair loops (the same premise the kernels rely
on) on every golden scene, at the default band and at a wider one that
puts more checks in the band.
"""
import numpy as np
import pytest

from conftest import GOLDEN_NAMES, load_golden
from gpuprm_b200 import scenes
import oracle as O

COUNTS = {"config1": 4000, "box4": 4000, "hull6": 1500, "wall7": 150}


@pytest.mark.parametrize("name", GOLDEN_NAMES)
@pytest.mark.parametrize("band", [1e-5, 1e-3])
def test_fp64_code_over_the_band_range_equals_the_full_check(name, band):
    sc, _ = load_golden(name)
    orc = O.Oracle(sc)
    q = scenes.uniform_configs(sc, COUNTS[name], 31).astype(np.float32)
    code32, margin, inband = orc.check_configs(q, O.FP32 | O.DEVICE_TRIG, band)
    lo, hi, c32 = orc.band_pair_range(q, O.DEVICE_TRIG, band)
    np.testing.assert_array_equal(c32, code32)
    full64, _, _ = orc.check_configs(q, O.FP64, band)
    sel = np.nonzero(inband)[0]
    assert len(sel) > 0, "no check in the band"
    assert np.all(lo[sel] < hi[sel]) and np.all(hi[sel] <= len(sc.pair_from))
    # a free check decided outside the band has no pair within it
    free_out = (code32 == 0) & ~inband
    assert np.all(lo[free_out] >= hi[free_out])
    ranged64 = orc.check_configs64_range(q[sel], lo[sel], hi[sel])
    np.testing.assert_array_equal(ranged64, full64[sel])
    # the range is usually far shorter than the pair list
    if len(sc.pair_from) > 100:
        assert np.mean(hi[sel] - lo[sel]) < 0.8 * len(sc.pair_from)
