"""Verdict parity of a checker's results with the reference's, by band class.

TEST INFRASTRUCTURE ONLY (tests/ and the bench's CPU legs).  The product
never imports it.

The bar the checker is held to: for every check whose FP32 separation
margin lies outside the band (|margin| >= band, not stopped by the
iteration cap), its free / not-free verdict equals the reference CPU
checker's; every check inside the band is recomputed in FP64 and its
verdict equals the FP64 oracle's.  For an edge (verdict = "some step is not
free", robotconfigspace.cpp:378-465, 694-705) the oracle's classes are
(orc_edge_classify):
  1  some step collides outside the band   -> every correct checker: not free
  0  every step is free outside the band   -> free
  2  otherwise: decided inside the band    -> the FP32 + FP64-band verdict
"""
from __future__ import annotations

import numpy as np


def verdict_parity(got: np.ndarray, ref: np.ndarray, cls: np.ndarray, band_res: np.ndarray,
                   inband_steps: np.ndarray | None = None) -> dict:
    """got: the checker's codes (nonzero = not free); ref: the reference
    CPU checker's codes for the same items; cls, band_res: the oracle's
    classes and FP32 + FP64-band codes.  Returns the counts of the parity
    object (all mismatch counts must be 0)."""
    got_v = np.asarray(got) != 0
    ref_v = np.asarray(ref) != 0
    band_v = np.asarray(band_res) != 0
    cls = np.asarray(cls)
    out_band = cls != 2
    cls_v = cls == 1
    d = {
        "checked": int(got_v.size),
        "not_free": int(got_v.sum()),
        "in_band": int((~out_band).sum()),
        # the headline bar: outside the band the checker agrees with the reference
        "mismatches_outside_band": int((out_band & (got_v != ref_v)).sum()),
        # inside the band the checker agrees with the FP64 oracle
        "mismatches_in_band_vs_fp64_oracle": int((~out_band & (got_v != band_v)).sum()),
        # the classification itself against the reference (pins the oracle's classes)
        "reference_vs_class_outside_band": int((out_band & (ref_v != cls_v)).sum()),
        # informational: FP32 reference and FP64 verdicts may differ inside the band
        "in_band_reference_differs": int((~out_band & (got_v != ref_v)).sum()),
    }
    if inband_steps is not None:
        d["in_band_steps"] = int(np.asarray(inband_steps).sum())
    return d


def parity_ok(d: dict) -> bool:
    return (d["mismatches_outside_band"] == 0 and d["mismatches_in_band_vs_fp64_oracle"] == 0
            and d["reference_vs_class_outside_band"] == 0)
