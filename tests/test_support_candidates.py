"""Support candidate lists of the fast path (host logic, no GPU).

The fast exact test (GPRM_MODE_FAST) finds a polytope's support vertex
along a direction as the maximum over the candidate list of the
direction's bin (dir_bin: a cube face and a 3 x 3 cell of it, the cell
borders at m (-1 + 2k/3), m the largest |component|).  The lists
are built on the host from each vertex's normal cone; the property that
makes the search exact is that, for every direction, the largest dot
product over the list equals the largest over all the polytope's vertices
(up to float rounding).  Checked on every polytope of the golden scenes
(the reference's config1 among them) for seeded random directions, with
bins computed in float32 exactly as the kernel computes them.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN_NAMES, load_golden
from gpuprm_b200.configspace import RobotConfigspace

BINS = 54


def dir_bin(d):
    """The kernel's dir_bin in float32 (same comparisons and rounding)."""
    x, y, z = (np.float32(c) for c in d)
    ax, ay, az = abs(x), abs(y), abs(z)
    if ax >= ay and ax >= az:
        face, m, u, v = (1 if x < 0 else 0), ax, y, z
    elif ay >= az:
        face, m, u, v = (3 if y < 0 else 2), ay, z, x
    else:
        face, m, u, v = (5 if z < 0 else 4), az, x, y
    iu = iv = 0
    for k in range(1, 3):
        c = np.float32(np.float32(-1.0) + np.float32(2.0) * np.float32(k) / np.float32(3.0))
        t = np.float32(m * c)
        iu += int(u > t)
        iv += int(v > t)
    return (face * 3 + iu) * 3 + iv


def candidates(cs, k, b):
    buf = (C.c_int * 128)()
    n = cs.lib.gprm_debug_support_candidates(cs.h, k, b, buf, 128)
    assert n > 0
    return np.array(buf[:n])


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_candidate_lists_contain_the_support(name):
    sc, z = load_golden(name)
    cs = RobotConfigspace(sc, dq=float(z["dq"]))
    rng = np.random.default_rng(5)
    sizes = []
    for k, poly in enumerate(sc.polys):
        V = np.asarray(poly.vertices, np.float64)
        lists = [candidates(cs, k, b) for b in range(BINS)]
        sizes += [len(l) for l in lists]
        for l in lists:
            assert np.all(np.diff(l) > 0) and l[0] >= 0 and l[-1] < len(V)
        D = rng.normal(size=(300, 3)).astype(np.float32)
        # directions on cell and face borders too: a component equal to a
        # third of another, or two equal components
        D[:20, 1] = D[:20, 0] / 3
        D[20:40, 2] = -D[20:40, 0]
        for d in D:
            dots = V @ d.astype(np.float64)
            best = dots.max()
            cand = dots[lists[dir_bin(d)]].max()
            scale = np.abs(V).max() * np.abs(d).max() + 1e-30
            assert cand >= best - 1e-6 * scale, (name, k, d)
    # far fewer candidates than vertices on average
    n_avg = np.mean([p.n for p in sc.polys])
    assert np.mean(sizes) < 0.5 * n_avg, (np.mean(sizes), n_avg)
