"""B200 configuration-space collision checker (GPUPRM's hot path).

The checking itself lives in libgprm_b200.so (hand-written sm_100a CUDA
behind a C ABI, include/gprm_b200.h); this package holds the Python mirror
of the reference's ``RobotConfigspace`` interface, the seeded scene
generators and the build step.
"""
from ._abi import (GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT, GPRM_MODE_FAST,  # noqa: F401
                   GPRM_MODE_FP32, GPRM_MODE_FP64_BAND, load_library)

__all__ = ["load_library", "GPRM_MODE_FP32", "GPRM_MODE_FP64_BAND", "GPRM_MODE_FAST", "GPRM_EDGES_EARLY_EXIT",
           "GPRM_EDGES_ALL_STEPS"]
