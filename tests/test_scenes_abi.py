"""Scene generators, the config-directory format and the C ABI surface (CPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from gpuprm_b200 import _abi, scenes
from gpuprm_b200.configspace import GprmError, RobotConfigspace


@pytest.mark.parametrize("kind", ["box4", "hull6", "mixed"])
def test_generators_valid_and_seeded(kind):
    a = scenes.make_scene(kind, 5)
    b = scenes.make_scene(kind, 5)
    a.validate()
    assert a.sumn == b.sumn
    for pa, pb in zip(a.polys, b.polys):
        np.testing.assert_array_equal(pa.vertices, pb.vertices)
        np.testing.assert_array_equal(pa.dest, pb.dest)
    for p in a.polys:
        # adjacency is symmetric and has no self loops
        for v in range(p.n):
            nb = p.dest[p.dsp[v]:p.dsp[v] + p.cnt[v]]
            assert v not in nb
            for u in nb:
                assert v in p.dest[p.dsp[u]:p.dsp[u] + p.cnt[u]]


def test_wall7_keeps_slot_open():
    sc = scenes.make_wall7(2, num_obstacles=64)
    gap = sc.meta["gap"]
    for p, s in zip(sc.polys, sc.sys):
        if s == 0:
            z = p.vertices[:, 2]
            assert z.min() >= 0.3 + gap / 2 - 1e-6 or z.max() <= 0.3 - gap / 2 + 1e-6


def test_config_dir_roundtrip(tmp_path):
    sc = scenes.make_hull6(3, num_obstacles=10)
    d = scenes.write_config_dir(sc, str(tmp_path / "scene"))
    back = scenes.read_config_dir(d)
    assert back.ndof == sc.ndof and back.num_pairs == sc.num_pairs
    for pa, pb in zip(sc.polys, back.polys):
        np.testing.assert_array_equal(pa.vertices, pb.vertices)
        np.testing.assert_array_equal(pa.dsp, pb.dsp)
        np.testing.assert_array_equal(pa.cnt, pb.cnt)
        np.testing.assert_array_equal(pa.dest, pb.dest)
    np.testing.assert_array_equal(sc.pair_from, back.pair_from)


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "gprm_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gprm_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load_library()
    names = header_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    declared = {n for n, _, _ in _abi.SIGNATURES}
    assert set(names) == declared


def _desc_holder(sc):
    return _abi.DescHolder(sc)


def _create(sc):
    lib = _abi.load_library()
    d = _desc_holder(sc)
    h = C.c_void_p()
    st = lib.gprm_create(d.ref(), 0.02, 0, C.byref(h))
    msg = lib.gprm_last_error(None).decode()
    if st == 0:
        lib.gprm_destroy(h)
    return st, msg


def test_create_accepts_valid_scene():
    st, _ = _create(scenes.make_box4(1))
    assert st == 0


@pytest.mark.parametrize("corrupt, expect", [
    ("cnt0", "cnt"), ("dest_oob", "dest"), ("n_too_big", "n="), ("pairs_unsorted", "sorted"),
    ("sys_oob", "sys"), ("pair_oob", "pair"), ("vertex_nan", "finite"),
])
def test_create_rejects_corrupt_scene(corrupt, expect):
    """Host-made faults: every corrupt CRS index is caught before any upload."""
    sc = scenes.make_box4(2)
    p = sc.polys[0]
    if corrupt == "cnt0":
        p.cnt[3] = 0
    elif corrupt == "dest_oob":
        p.dest[5] = p.n + 3
    elif corrupt == "n_too_big":
        big = np.random.default_rng(0).normal(size=(150, 3))
        big /= np.linalg.norm(big, axis=1, keepdims=True)
        v = np.concatenate([big] * 1).astype(np.float32)
        sc.polys[0] = scenes.Polytope(v, np.zeros(150, np.int32), np.ones(150, np.int32),
                                      np.zeros(1, np.int32))
    elif corrupt == "pairs_unsorted":
        sc.pair_from = sc.pair_from[::-1].copy()
        sc.pair_to = sc.pair_to[::-1].copy()
    elif corrupt == "sys_oob":
        sc.sys = sc.sys.copy()
        sc.sys[-1] = 9
    elif corrupt == "pair_oob":
        sc.pair_to = sc.pair_to.copy()
        sc.pair_to[0] = 1000
    elif corrupt == "vertex_nan":
        p.vertices = p.vertices.copy()
        p.vertices[0, 1] = np.nan
    st, msg = _create(sc)
    assert st in (_abi.GPRM_OK - 1, -2), (st, msg)
    assert expect in msg


def test_create_from_dir_and_queries(tmp_path):
    sc = scenes.make_box4(6)
    d = scenes.write_config_dir(sc, str(tmp_path / "c"))
    cs = RobotConfigspace(d, dq=0.02, nbuf=64)
    assert cs.dim() == 4
    assert abs(cs.deltaq() - 0.02) < 1e-9
    assert cs.min(0) == np.float32(-np.pi) and cs.max(3) == np.float32(np.pi)
    # check_boundaries runs on the host (robotconfigspace.cpp:780-802)
    q = np.array([0.0, 0.0, 4.0, 0.0], np.float32)
    assert cs.check_boundaries(q) == 1
    assert cs.check_boundaries(np.zeros(4, np.float32)) == 0
    with pytest.raises(GprmError):
        RobotConfigspace(d, dq=0.02, nbuf=64, ndof=5)
    with pytest.raises(GprmError):
        RobotConfigspace(str(tmp_path / "missing"), dq=0.02, nbuf=64, ndof=4)


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_queries_without_gpu_fail_cleanly():
    cs = RobotConfigspace(scenes.make_box4(1), dq=0.02)
    with pytest.raises(GprmError) as e:
        cs.init()
    assert e.value.status == -4
    with pytest.raises(GprmError) as e:
        cs.indicator(np.zeros(4, np.float32))
    assert e.value.status == -6   # not initialised


def test_edge_split_arguments_checked_on_host():
    cs = RobotConfigspace(scenes.make_box4(1), dq=0.02)
    for bad in ((-1, 2), ((1 << 22) + 1, 2), (100, 0)):
        with pytest.raises(GprmError) as e:
            cs.set_edge_split(*bad)
        assert e.value.status == -1
    cs.set_edge_split(0)
    cs.set_edge_split(16384, 4)
    cs.set_edge_split(1 << 22, 2)


REF_LIB_DIR = "/root/reference/prm/src/lib"


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_LIB_DIR, "prm", "configspace.hpp")),
                    reason="the reference's Configspace header is only present where the reference is")
def test_cpp_shim_implements_reference_interface(tmp_path):
    """include/gprm_configspace.hpp compiles against the reference's own
    Configspace<ndof> (every pure virtual overridden) and links against
    libgprm_b200.so."""
    import subprocess
    src = tmp_path / "shim.cpp"
    src.write_text(
        '#include <prm/configspace.hpp>\n#include "gprm_configspace.hpp"\n'
        "int main(int argc, char** argv) {\n"
        "  if (argc < 2) return 0;\n"
        "  B200RobotConfigspace<4> s(argv[1], 0.01f, 64);\n"
        "  Configspace<4>* cs = &s;\n"
        "  return cs->dim() == 4 ? 0 : 1;\n}\n")
    lib_dir = os.path.join(ROOT, "gpuprm_b200")
    r = subprocess.run(["g++", "-std=c++14", "-I", REF_LIB_DIR, "-I", os.path.join(ROOT, "include"), str(src),
                        "-L", lib_dir, "-lgprm_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(tmp_path / "shim")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    sc = scenes.make_box4(1)
    d = scenes.write_config_dir(sc, str(tmp_path / "scene"))
    assert subprocess.run([str(tmp_path / "shim"), d]).returncode == 0
