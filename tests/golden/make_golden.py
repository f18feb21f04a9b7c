"""Generates the golden fixtures in this directory from the reference itself.

Each fixture (.npz) holds one scene (arrays in the gprm_scene_desc layout),
seeded vertex configurations and edges, and the verdicts that GPUPRM's own
CPU checker returns for them: RobotConfigspace<ndof>::indicator(q) per
configuration (robotconfigspace.cpp:313-346) and indicator2 per edge, which
leaves the code of the last colliding step (robotconfigspace.cpp:458,
694-705).  The reference checker is oracle/_ref/libgprm_ref.so, compiled
from the reference sources by oracle/Makefile; this script therefore runs
only where the reference tree is present.

Scenes: the reference's own prm/config1 (4-DOF, 13 polytopes, 44 pairs),
and generated box4 / hull6 / wall7 scenes.

    python tests/golden/make_golden.py [--reference /root/reference]
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from gpuprm_b200 import scenes  # noqa: E402
from oracle import RefChecker  # noqa: E402

SCENE_KEYS = ["a", "alpha", "q0", "d0", "types", "mins", "maxs", "sys", "pair_from", "pair_to"]


def scene_arrays(sc: scenes.Scene) -> dict:
    poly_n, poly_m, verts, dsp, cnt, dest = sc.flat()
    out = {k: getattr(sc, k) for k in SCENE_KEYS}
    out.update(ndof=np.int32(sc.ndof), poly_n=poly_n, poly_m=poly_m, verts=verts, dsp=dsp, cnt=cnt,
               dest=dest)
    return out


def scene_from_npz(z) -> scenes.Scene:
    """Rebuilds the Scene stored by scene_arrays()."""
    polys = []
    vo = mo = 0
    for n, m in zip(z["poly_n"], z["poly_m"]):
        n, m = int(n), int(m)
        polys.append(scenes.Polytope(z["verts"][vo:vo + n], z["dsp"][vo:vo + n], z["cnt"][vo:vo + n],
                                     z["dest"][mo:mo + m]))
        vo += n
        mo += m
    return scenes.Scene(int(z["ndof"]), z["a"], z["alpha"], z["q0"], z["d0"], z["types"], z["mins"],
                        z["maxs"], polys, z["sys"], z["pair_from"], z["pair_to"], str(z["name"]))


CASES = [
    # name, scene factory, n configs, config range, n edges, edge max length, dq
    ("config1", None, 4096, (-3.5, 5.0), 512, 0.5, 0.01),
    ("box4", lambda: scenes.make_box4(1), 4096, None, 512, 0.5, 0.02),
    ("hull6", lambda: scenes.make_hull6(2), 2048, None, 256, 0.7, 0.01),
    ("wall7", lambda: scenes.make_wall7(3, num_obstacles=96), 1024, None, 128, 0.6, 0.01),
]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    for name, factory, nq, qrange, ne, elen, dq in CASES:
        if factory is None:
            sc = scenes.read_config_dir(os.path.join(args.reference, "prm", "config1"), "config1")
        else:
            sc = factory()
        seed = {"config1": 11, "box4": 12, "hull6": 13, "wall7": 14}[name]
        if qrange is None:
            q = scenes.uniform_configs(sc, nq, seed)
        else:
            q = scenes.uniform_configs(sc, nq, seed, qrange[0], qrange[1])
        qs, qe = scenes.random_edges(sc, ne, seed + 100, elen)
        ref = RefChecker(sc, dq=dq, nbuf=4096)
        codes = ref.check_configs(q)
        eres = ref.check_edges(qs, qe)
        out = scene_arrays(sc)
        out.update(name=np.array(name), q=q, codes=codes.astype(np.int8), qs=qs, qe=qe,
                   edge_res=eres.astype(np.int8), dq=np.float32(dq))
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {nq} configs (free {np.mean(codes == 0):.2f}), {ne} edges "
              f"(free {np.mean(eres == 0):.2f}) -> {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
