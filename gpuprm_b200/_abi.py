"""ctypes view of the C ABI declared in include/gprm_b200.h."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libgprm_b200.so")

GPRM_OK = 0
GPRM_MODE_FP32 = 0
GPRM_MODE_FP64_BAND = 1
GPRM_MODE_FAST = 2
GPRM_EDGES_EARLY_EXIT = 0
GPRM_EDGES_ALL_STEPS = 1
GPRM_MLP_INFER_TCGEN05 = 0
GPRM_MLP_INFER_TRAINING_GEMM = 1
GPRM_MLP_INFER_TCGEN05_LAYERS = 2
GPRM_MLP_TRAIN_TCGEN05 = 0
GPRM_MLP_TRAIN_MMA_SYNC = 1
GPRM_MAX_DOF = 7
GPRM_MAX_VERTICES = 100
GPRM_NOALLOC_MAX_CONFIGS = 65536


class SceneDesc(C.Structure):
    _fields_ = [
        ("ndof", C.c_int),
        ("dh_a", C.POINTER(C.c_float)),
        ("dh_alpha", C.POINTER(C.c_float)),
        ("dh_q", C.POINTER(C.c_float)),
        ("dh_d", C.POINTER(C.c_float)),
        ("dh_types", C.POINTER(C.c_int)),
        ("mins", C.POINTER(C.c_float)),
        ("maxs", C.POINTER(C.c_float)),
        ("num_polytopes", C.c_int),
        ("poly_n", C.POINTER(C.c_int)),
        ("poly_m", C.POINTER(C.c_int)),
        ("vertices", C.POINTER(C.c_float)),
        ("dsp", C.POINTER(C.c_int)),
        ("cnt", C.POINTER(C.c_int)),
        ("dest", C.POINTER(C.c_int)),
        ("sys", C.POINTER(C.c_int)),
        ("num_pairs", C.c_int),
        ("pair_from", C.POINTER(C.c_int)),
        ("pair_to", C.POINTER(C.c_int)),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("vertex_checks", C.c_int64),
        ("edge_steps_nominal", C.c_int64),
        ("edge_steps_executed", C.c_int64),
        ("band_rechecks", C.c_int64),
        ("band_flips", C.c_int64),
        ("launches", C.c_int64),
        ("pairs_certified", C.c_int64),
        ("pairs_tested", C.c_int64),
        ("band_overflow_items", C.c_int64),
    ]


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


class DescHolder:
    """A ``SceneDesc`` plus the numpy arrays it points into (kept alive)."""

    def __init__(self, scene):
        f32 = lambda x: np.ascontiguousarray(np.asarray(x, np.float32))
        i32 = lambda x: np.ascontiguousarray(np.asarray(x, np.int32))
        poly_n, poly_m, verts, dsp, cnt, dest = scene.flat()
        self.arrays = dict(
            a=f32(scene.a), alpha=f32(scene.alpha), q=f32(scene.q0), d=f32(scene.d0),
            types=i32(scene.types), mins=f32(scene.mins), maxs=f32(scene.maxs),
            poly_n=i32(poly_n), poly_m=i32(poly_m), verts=f32(verts.reshape(-1)),
            dsp=i32(dsp), cnt=i32(cnt), dest=i32(dest), sys=i32(scene.sys),
            pf=i32(scene.pair_from), pt=i32(scene.pair_to))
        A = self.arrays
        self.desc = SceneDesc(
            scene.ndof, fptr(A["a"]), fptr(A["alpha"]), fptr(A["q"]), fptr(A["d"]),
            iptr(A["types"]), fptr(A["mins"]), fptr(A["maxs"]), scene.num_polys,
            iptr(A["poly_n"]), iptr(A["poly_m"]), fptr(A["verts"]), iptr(A["dsp"]),
            iptr(A["cnt"]), iptr(A["dest"]), iptr(A["sys"]), scene.num_pairs,
            iptr(A["pf"]), iptr(A["pt"]))

    def ref(self):
        return C.byref(self.desc)


_P = C.c_void_p
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)

# (name, restype, argtypes) of every exported symbol
SIGNATURES = [
    ("gprm_create", C.c_int, [C.POINTER(SceneDesc), C.c_float, C.c_int, C.POINTER(_P)]),
    ("gprm_create_from_dir", C.c_int, [C.c_char_p, C.c_int, C.c_float, C.c_int, C.POINTER(_P)]),
    ("gprm_init", C.c_int, [_P, C.c_int, C.c_int]),
    ("gprm_destroy", None, [_P]),
    ("gprm_last_error", C.c_char_p, [_P]),
    ("gprm_set_mode", C.c_int, [_P, C.c_int]),
    ("gprm_set_edge_policy", C.c_int, [_P, C.c_int]),
    ("gprm_set_edge_split", C.c_int, [_P, C.c_int, C.c_int]),
    ("gprm_set_band", C.c_int, [_P, C.c_float]),
    ("gprm_get_stats", C.c_int, [_P, C.POINTER(Stats)]),
    ("gprm_indicator", C.c_int, [_P, _F, _I]),
    ("gprm_indicator_batch", C.c_int, [_P, _F, _I, C.c_int, C.c_int]),
    ("gprm_indicator2", C.c_int, [_P, _F, _F, _I, C.c_int, C.c_int]),
    ("gprm_indicator2_compressed", C.c_int, [_P, _F, C.c_int, _F, _I, _I, _I, C.c_int]),
    ("gprm_indicator2_async", C.c_int, [_P, _F, _F, _I, C.c_int, C.c_int, _I]),
    ("gprm_indicator2_wait", C.c_int, [_P, C.c_int]),
    ("gprm_check_boundaries", C.c_int, [_P, _F, _I, C.c_int, C.c_int]),
    ("gprm_check_boundaries1", C.c_int, [_P, _F, _I]),
    ("gprm_min", C.c_float, [_P, C.c_int]),
    ("gprm_max", C.c_float, [_P, C.c_int]),
    ("gprm_deltaq", C.c_float, [_P]),
    ("gprm_dim", C.c_int, [_P]),
    ("gprm_indicator_batch_device", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    ("gprm_indicator2_device", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    ("gprm_indicator_batch_device_noalloc", C.c_int,
     [_P, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    ("gprm_mlp_create", C.c_int, [C.c_int, C.c_ulonglong, C.POINTER(_P)]),
    ("gprm_mlp_destroy", None, [_P]),
    ("gprm_mlp_last_error", C.c_char_p, [_P]),
    ("gprm_mlp_num_params", C.c_longlong, [_P]),
    ("gprm_mlp_get_params", C.c_int, [_P, _F]),
    ("gprm_mlp_set_params", C.c_int, [_P, _F]),
    ("gprm_mlp_predict", C.c_int, [_P, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    ("gprm_mlp_gradients", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_int, C.c_int, _F, _F]),
    ("gprm_mlp_adam_step", C.c_int, [_P, C.c_float]),
    ("gprm_mlp_set_inference", C.c_int, [_P, C.c_int]),
    ("gprm_mlp_set_training", C.c_int, [_P, C.c_int]),
    ("gprm_mlp_device_status", C.c_int, [_P, C.POINTER(C.c_uint)]),
    ("gprm_mlp_set_wait_budget", C.c_int, [_P, C.c_longlong]),
    ("gprm_mlp_train", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                 C.c_float, _F]),
    ("gprm_debug_fk", C.c_int, [_P, _F, _F]),
    ("gprm_device_sm_count", C.c_int, [_P]),
    ("gprm_debug_support_candidates", C.c_int, [_P, C.c_int, C.c_int, _I, C.c_int]),
    ("gprm_debug_set_queue_capacity", C.c_int, [_P, C.c_uint]),
    ("gprm_debug_fail_device_alloc", None, [C.c_longlong]),
    ("gprm_set_launch", C.c_int, [_P, C.c_int, C.c_int, C.c_int]),
    ("gprm_set_launch_shape", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("gprm_get_launch", C.c_int, [_P, C.c_int, _I, _I, _I]),
    ("gprm_profile_enable", C.c_int, [_P, C.c_int]),
    ("gprm_profile_read", C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("gprm_measure_fp32_peak", C.c_int, [C.POINTER(C.c_double)]),
    ("gprm_batch_create", C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(_P)]),
    ("gprm_batch_destroy", None, [_P]),
    ("gprm_batch_last_error", C.c_char_p, [_P]),
    ("gprm_batch_set_layout", C.c_int, [_P, C.c_int, C.POINTER(C.c_longlong), C.c_longlong]),
    ("gprm_batch_indicator_device", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]),
    ("gprm_batch_indicator2_device", C.c_int,
     [_P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]),
    ("gprm_batch_capture", C.c_int, [_P, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong]),
    ("gprm_batch_replay", C.c_int, [_P, C.c_int, C.c_void_p]),
    ("gprm_batch_set_launch", C.c_int, [_P, C.c_int, C.c_int]),
    ("gprm_batch_get_launch", C.c_int, [_P, C.c_int, _I, _I]),
    ("gprm_batch_set_launch_shape", C.c_int, [_P, C.c_int, C.c_int, C.c_int]),
    ("gprm_batch_get_launch_shape", C.c_int, [_P, C.c_int, _I, _I, _I]),
    ("gprm_batch_get_tune_table", C.c_int, [_P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            _I]),
    ("gprm_batch_set_solo_threshold", C.c_int, [_P, C.c_int, C.c_longlong]),
    ("gprm_batch_get_solo_threshold", C.c_int, [_P, C.c_int, C.POINTER(C.c_longlong), _I]),
    ("gprm_batch_autotune", C.c_int, [_P, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int,
                                      _I, _F]),
    ("gprm_batch_get_stats", C.c_int, [_P, C.POINTER(Stats)]),
    ("gprm_nbr_create", C.c_int, [C.c_int, C.POINTER(_P)]),
    ("gprm_nbr_destroy", None, [_P]),
    ("gprm_nbr_last_error", C.c_char_p, [_P]),
    ("gprm_nbr_build", C.c_int, [_P, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_void_p]),
    ("gprm_nbr_radius", C.c_int, [_P, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
    ("gprm_nbr_knn", C.c_int, [_P, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                               C.c_void_p]),
    ("gprm_nbr_redo_count", C.c_int, [_P, _I]),
    ("gprm_sample_near", C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_float,
                                   C.c_ulonglong, C.c_longlong, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                   C.c_void_p]),
    ("gprm_sample_near_blocks", C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                          C.c_void_p, C.c_int, C.c_float, C.c_ulonglong, C.c_longlong, C.c_int,
                                          C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("gprm_graph_create", C.c_int, [C.POINTER(_P)]),
    ("gprm_graph_destroy", None, [_P]),
    ("gprm_graph_last_error", C.c_char_p, [_P]),
    ("gprm_graph_components", C.c_int, [_P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    ("gprm_graph_forest", C.c_int, [_P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, _I, C.c_void_p]),
    ("gprm_graph_path_lengths", C.c_int, [_P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gprm_graph_path_write", C.c_int, [_P, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gprm_graph_sssp", C.c_int, [_P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                  C.c_void_p, C.c_void_p, _I, C.c_void_p]),
]

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libgprm_b200.so; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(the collision checker has no CPU fallback)")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
