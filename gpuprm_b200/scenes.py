"""Seeded scene generators and the reference's on-disk scene format.

A *scene* is what ``RobotConfigspace<ndof>`` loads from a config directory
(prm/src/lib/robotspace/robotconfigspace.cpp:101-208): modified-DH arm
parameters, joint bounds, a list of convex polytopes (vertices plus a CRS
vertex-adjacency graph), the frame ("sys") each polytope is attached to, and
the list of polytope pairs to test, sorted by ``from``.

Convex hulls are built with Qhull (scipy.spatial.ConvexHull); the hull's
triangle edges become the CRS adjacency and points that are not hull vertices
are dropped, which is what the reference's MATLAB tooling does
(prm/matlab/lib/polygen2.m, polywrite.m).  Every vertex therefore has at least
one neighbour and no polytope has more than 100 vertices, the two conditions
``RobotConfigspace::construct`` asserts (robotconfigspace.cpp:44-51).

Workloads (all from one seed):

* ``box4``    4-DOF arm, box links 0.3x0.05x0.05 m, 16 obstacle boxes.
* ``hull6``   6-DOF arm, links = hull of 16 points on an ellipsoid
              (0.15/0.04/0.04 m), 64 obstacles = hull of 12-32 points in a
              box of side U[0.05,0.3] m.
* ``wall7``   7-DOF arm, 8 links of 32-vertex hulls, 512 obstacles of 8-64
              points in 6 Gaussian clusters forming two walls with a 0.12 m gap.
* ``mixed``   one scene of a many-problem batch: DOF in {4..7}, obstacle count
              log-uniform in [8,128], obstacles as in ``hull6``.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

MAX_VERTICES = 100  # robotconfigspace.cpp:50 (max_vertices_number, collision4.h:19)


@dataclass
class Polytope:
    vertices: np.ndarray  # (n, 3) float32, body frame
    dsp: np.ndarray       # (n,) int32, CRS offsets into dest
    cnt: np.ndarray       # (n,) int32, neighbour counts (all > 0)
    dest: np.ndarray      # (m,) int32, local neighbour indices

    @property
    def n(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def m(self) -> int:
        return int(self.dest.shape[0])


@dataclass
class Scene:
    ndof: int
    a: np.ndarray        # (ndof,) float32
    alpha: np.ndarray    # (ndof,) float32
    q0: np.ndarray       # (ndof,) float32  (theta of prismatic joints)
    d0: np.ndarray       # (ndof,) float32  (d of revolute joints)
    types: np.ndarray    # (ndof,) int32, 0 revolute, 1 prismatic
    mins: np.ndarray     # (ndof,) float32
    maxs: np.ndarray     # (ndof,) float32
    polys: List[Polytope]
    sys: np.ndarray      # (N,) int32, frame of each polytope (0 = world)
    pair_from: np.ndarray  # (M,) int32, sorted ascending
    pair_to: np.ndarray    # (M,) int32
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def num_polys(self) -> int:
        return len(self.polys)

    @property
    def num_pairs(self) -> int:
        return int(self.pair_from.shape[0])

    @property
    def sumn(self) -> int:
        return sum(p.n for p in self.polys)

    def flat(self):
        """Concatenated arrays in the layout of ``gprm_scene_desc``."""
        poly_n = np.array([p.n for p in self.polys], np.int32)
        poly_m = np.array([p.m for p in self.polys], np.int32)
        verts = np.ascontiguousarray(np.concatenate([p.vertices for p in self.polys]).astype(np.float32))
        dsp = np.ascontiguousarray(np.concatenate([p.dsp for p in self.polys]).astype(np.int32))
        cnt = np.ascontiguousarray(np.concatenate([p.cnt for p in self.polys]).astype(np.int32))
        dest = np.ascontiguousarray(np.concatenate([p.dest for p in self.polys]).astype(np.int32))
        return poly_n, poly_m, verts, dsp, cnt, dest

    def validate(self) -> None:
        assert self.sys.shape[0] == len(self.polys)
        assert np.all(np.diff(self.sys) >= 0), "polytopes must be sorted by sys"
        assert np.all(np.diff(self.pair_from) >= 0), "pairs must be sorted by from"
        assert self.sys.max() <= self.ndof
        for p in self.polys:
            assert 0 < p.n <= MAX_VERTICES
            assert np.all(p.cnt > 0)
            assert np.all(p.dsp + p.cnt <= p.m)
            assert np.all((p.dest >= 0) & (p.dest < p.n))


# --------------------------------------------------------------------------
# convex hull -> CRS polytope
# --------------------------------------------------------------------------

def hull_polytope(points: np.ndarray) -> Polytope:
    """Convex hull of ``points`` as a polytope with triangle-edge adjacency.

    Vertices are the hull vertices in ascending order of their index in
    ``points``; each vertex lists its neighbours in ascending order.
    """
    from scipy.spatial import ConvexHull

    pts = np.asarray(points, np.float64)
    hull = ConvexHull(pts)
    vids = np.array(sorted(int(v) for v in hull.vertices))
    remap = {int(v): i for i, v in enumerate(vids)}
    nbr = [set() for _ in vids]
    for tri in hull.simplices:
        t = [remap[int(x)] for x in tri]
        for i in range(3):
            a, b = t[i], t[(i + 1) % 3]
            if a != b:
                nbr[a].add(b)
                nbr[b].add(a)
    cnt = np.array([len(s) for s in nbr], np.int32)
    dsp = np.zeros_like(cnt)
    dsp[1:] = np.cumsum(cnt)[:-1]
    dest = np.array([j for s in nbr for j in sorted(s)], np.int32)
    verts = pts[vids].astype(np.float32)
    poly = Polytope(verts, dsp, cnt, dest)
    assert poly.n <= MAX_VERTICES and np.all(cnt > 0)
    return poly


def box_points(lx: float, ly: float, lz: float, x0: float = 0.0) -> np.ndarray:
    """The 8 corners of an axis-aligned box [x0,x0+lx] x [-ly/2,ly/2] x [-lz/2,lz/2]."""
    xs = [x0, x0 + lx]
    ys = [-ly / 2, ly / 2]
    zs = [-lz / 2, lz / 2]
    return np.array([[x, y, z] for x in xs for y in ys for z in zs], np.float64)


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform random rotation (Shoemake's uniform quaternion)."""
    u1, u2, u3 = rng.random(3)
    a = math.sqrt(1 - u1)
    b = math.sqrt(u1)
    x, y = a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2)
    z, w = b * math.sin(2 * math.pi * u3), b * math.cos(2 * math.pi * u3)
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _centre_outside_ball(rng, lo=-1.0, hi=1.0, rmin=0.25) -> np.ndarray:
    while True:
        c = rng.uniform(lo, hi, 3)
        if np.linalg.norm(c) >= rmin:
            return c


def _arm(ndof: int, a: float = 0.3):
    alpha = np.array([(math.pi / 2) * (1 if i % 2 == 0 else -1) for i in range(ndof)], np.float32)
    return (np.full(ndof, a, np.float32), alpha, np.zeros(ndof, np.float32),
            np.zeros(ndof, np.float32), np.zeros(ndof, np.int32))


def _pairs(num_obstacles: int, link_ids: List[int], link_sys: List[int]):
    """Every obstacle against every link, then link against non-adjacent link."""
    pf, pt = [], []
    for o in range(num_obstacles):
        for l in link_ids:
            pf.append(o)
            pt.append(l)
    for i, li in enumerate(link_ids):
        for j in range(i + 1, len(link_ids)):
            if abs(link_sys[j] - link_sys[i]) >= 2:
                pf.append(li)
                pt.append(link_ids[j])
    return np.array(pf, np.int32), np.array(pt, np.int32)


def _assemble(ndof, arm, obstacles, links, link_sys, name, meta, bound=math.pi):
    a, alpha, q0, d0, types = arm
    polys = list(obstacles) + list(links)
    nobs = len(obstacles)
    sys = np.array([0] * nobs + list(link_sys), np.int32)
    link_ids = list(range(nobs, nobs + len(links)))
    pf, pt = _pairs(nobs, link_ids, list(link_sys))
    sc = Scene(ndof, a, alpha, q0, d0, types,
               np.full(ndof, -bound, np.float32), np.full(ndof, bound, np.float32),
               polys, sys, pf, pt, name, meta)
    sc.validate()
    return sc


def make_box4(seed: int = 0, num_obstacles: int = 16) -> Scene:
    """4-DOF box arm with 16 random boxes (the reference's CPU-runnable case)."""
    rng = np.random.default_rng(seed)
    ndof = 4
    links = [hull_polytope(box_points(0.3, 0.05, 0.05)) for _ in range(ndof)]
    obstacles = []
    for _ in range(num_obstacles):
        side = rng.uniform(0.05, 0.2, 3)
        c = _centre_outside_ball(rng)
        R = random_rotation(rng)
        pts = box_points(side[0], side[1], side[2], -side[0] / 2) @ R.T + c
        obstacles.append(hull_polytope(pts))
    return _assemble(ndof, _arm(ndof), obstacles, links, list(range(1, ndof + 1)),
                     "box4", {"seed": seed})


def _ellipsoid_link(rng, npts=16, axes=(0.15, 0.04, 0.04)):
    while True:
        d = rng.normal(size=(npts, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        pts = d * np.array(axes) + np.array([axes[0], 0.0, 0.0])
        try:
            return hull_polytope(pts)
        except Exception:  # degenerate draw; resample
            continue


def _random_hull_obstacle(rng, npts_lo=12, npts_hi=32, side_lo=0.05, side_hi=0.3, centre=None):
    npts = int(rng.integers(npts_lo, npts_hi + 1))
    side = rng.uniform(side_lo, side_hi, 3)
    pts = rng.uniform(-0.5, 0.5, (npts, 3)) * side
    R = random_rotation(rng)
    c = _centre_outside_ball(rng) if centre is None else centre
    return hull_polytope(pts @ R.T + c)


def make_hull6(seed: int = 0, num_obstacles: int = 64, ndof: int = 6) -> Scene:
    """6-DOF ellipsoid-hull arm among 64 random hull obstacles."""
    rng = np.random.default_rng(seed)
    links = [_ellipsoid_link(rng) for _ in range(ndof)]
    obstacles = [_random_hull_obstacle(rng) for _ in range(num_obstacles)]
    return _assemble(ndof, _arm(ndof), obstacles, links, list(range(1, ndof + 1)),
                     f"hull{ndof}", {"seed": seed})


def make_mixed(seed: int) -> Scene:
    """One problem of the many-problem batch: DOF in {4..7}, 8-128 obstacles."""
    rng = np.random.default_rng(seed)
    ndof = int(rng.integers(4, 8))
    nobs = int(round(math.exp(rng.uniform(math.log(8), math.log(128)))))
    links = [_ellipsoid_link(rng) for _ in range(ndof)]
    obstacles = [_random_hull_obstacle(rng) for _ in range(nobs)]
    return _assemble(ndof, _arm(ndof), obstacles, links, list(range(1, ndof + 1)),
                     "mixed", {"seed": seed})


def make_wall7(seed: int = 0, num_obstacles: int = 512, gap: float = 0.12) -> Scene:
    """7-DOF arm (8 links incl. the base link) and two cluttered walls with a gap.

    Six Gaussian clusters (sigma 0.15 m) are centred on the plane x = 0.6; three
    lie above the slot |z - 0.3| < gap/2 and three below it.  Obstacle centres
    that would reach into the slot are redrawn, so the slot stays open.
    """
    rng = np.random.default_rng(seed)
    ndof = 7
    links = [_ellipsoid_link(rng, npts=32) for _ in range(ndof + 1)]
    link_sys = list(range(0, ndof + 1))
    slot_z = 0.3
    centres = []
    for side in (+1, -1):
        for yc in (-0.5, 0.0, 0.5):
            centres.append(np.array([0.6, yc, slot_z + side * (gap / 2 + 0.25)]))
    obstacles = []
    while len(obstacles) < num_obstacles:
        cc = centres[len(obstacles) % 6]
        c = cc + rng.normal(0.0, 0.15, 3) * np.array([0.3, 1.0, 1.0])
        above = cc[2] > slot_z
        npts = int(rng.integers(8, 65))
        side = rng.uniform(0.04, 0.12, 3)
        pts = rng.uniform(-0.5, 0.5, (npts, 3)) * side
        R = random_rotation(rng)
        world = pts @ R.T + c
        zmin, zmax = world[:, 2].min(), world[:, 2].max()
        if above and zmin < slot_z + gap / 2:
            continue
        if (not above) and zmax > slot_z - gap / 2:
            continue
        if np.linalg.norm(c) < 0.25:
            continue
        try:
            obstacles.append(hull_polytope(world))
        except Exception:
            continue
    return _assemble(ndof, _arm(ndof), obstacles, links, link_sys, "wall7",
                     {"seed": seed, "gap": gap})


def make_scene(kind: str, seed: int = 0) -> Scene:
    if kind == "box4":
        return make_box4(seed)
    if kind == "hull6":
        return make_hull6(seed)
    if kind == "wall7":
        return make_wall7(seed)
    if kind == "mixed":
        return make_mixed(seed)
    raise ValueError(f"unknown scene kind {kind!r}")


# --------------------------------------------------------------------------
# the reference's config-directory format (robotconfigspace.cpp:101-208)
# --------------------------------------------------------------------------

def _w(path, arr, dt):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.ascontiguousarray(np.asarray(arr, dt)).tofile(path)


def write_config_dir(scene: Scene, path: str) -> str:
    """Write ``scene`` so that ``RobotConfigspace<ndof>(path, dq, nbuf)`` loads it."""
    _w(os.path.join(path, "ndof.bin"), [scene.ndof], np.int32)
    _w(os.path.join(path, "dh", "a.bin"), scene.a, np.float32)
    _w(os.path.join(path, "dh", "alpha.bin"), scene.alpha, np.float32)
    _w(os.path.join(path, "dh", "q.bin"), scene.q0, np.float32)
    _w(os.path.join(path, "dh", "d.bin"), scene.d0, np.float32)
    _w(os.path.join(path, "dh", "types.bin"), scene.types, np.int32)
    _w(os.path.join(path, "mins.bin"), scene.mins, np.float32)
    _w(os.path.join(path, "maxs.bin"), scene.maxs, np.float32)
    _w(os.path.join(path, "polys", "N.bin"), [scene.num_polys], np.int32)
    _w(os.path.join(path, "polys", "sys.bin"), scene.sys, np.int32)
    _w(os.path.join(path, "pairs", "M.bin"), [scene.num_pairs], np.int32)
    _w(os.path.join(path, "pairs", "from.bin"), scene.pair_from, np.int32)
    _w(os.path.join(path, "pairs", "to.bin"), scene.pair_to, np.int32)
    for i, p in enumerate(scene.polys):
        d = os.path.join(path, "polys", f"poly{i}")
        _w(os.path.join(d, "size.bin"), [p.n, p.m], np.int32)
        _w(os.path.join(d, "vertices.bin"), p.vertices.reshape(-1), np.float32)
        _w(os.path.join(d, "dsp.bin"), p.dsp, np.int32)
        _w(os.path.join(d, "cnt.bin"), p.cnt, np.int32)
        _w(os.path.join(d, "dest.bin"), p.dest, np.int32)
    return path


def read_config_dir(path: str, name: str = "") -> Scene:
    """Load a scene written in the reference's config-directory format."""
    r = lambda p, dt: np.fromfile(os.path.join(path, p), dtype=dt)
    ndof = int(r("ndof.bin", np.int32)[0])
    N = int(r("polys/N.bin", np.int32)[0])
    M = int(r("pairs/M.bin", np.int32)[0])
    polys = []
    for i in range(N):
        n, m = (int(x) for x in r(f"polys/poly{i}/size.bin", np.int32)[:2])
        polys.append(Polytope(
            r(f"polys/poly{i}/vertices.bin", np.float32)[: 3 * n].reshape(n, 3),
            r(f"polys/poly{i}/dsp.bin", np.int32)[:n],
            r(f"polys/poly{i}/cnt.bin", np.int32)[:n],
            r(f"polys/poly{i}/dest.bin", np.int32)[:m]))
    return Scene(ndof,
                 r("dh/a.bin", np.float32)[:ndof], r("dh/alpha.bin", np.float32)[:ndof],
                 r("dh/q.bin", np.float32)[:ndof], r("dh/d.bin", np.float32)[:ndof],
                 r("dh/types.bin", np.int32)[:ndof],
                 r("mins.bin", np.float32)[:ndof], r("maxs.bin", np.float32)[:ndof],
                 polys, r("polys/sys.bin", np.int32)[:N],
                 r("pairs/from.bin", np.int32)[:M], r("pairs/to.bin", np.int32)[:M],
                 name or os.path.basename(os.path.normpath(path)))


# --------------------------------------------------------------------------
# seeded query generators
# --------------------------------------------------------------------------

def uniform_configs(scene: Scene, n: int, seed: int, lo: Optional[float] = None,
                    hi: Optional[float] = None) -> np.ndarray:
    """``n`` configurations uniform in [lo,hi]^ndof (default: the joint bounds), (n, ndof) float32."""
    rng = np.random.default_rng(seed)
    lo_ = scene.mins.astype(np.float64) if lo is None else np.full(scene.ndof, lo)
    hi_ = scene.maxs.astype(np.float64) if hi is None else np.full(scene.ndof, hi)
    return rng.uniform(lo_, hi_, (n, scene.ndof)).astype(np.float32)


def random_edges(scene: Scene, n: int, seed: int, max_len: float) -> tuple:
    """``n`` edges (qs, qe), each (n, ndof) float32: a uniform start and an end
    at a uniform distance in (0, max_len] along a uniform direction, clipped to
    the joint bounds."""
    rng = np.random.default_rng(seed)
    qs = rng.uniform(scene.mins, scene.maxs, (n, scene.ndof))
    d = rng.normal(size=(n, scene.ndof))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    qe = qs + d * rng.uniform(0, max_len, (n, 1))
    qe = np.clip(qe, scene.mins, scene.maxs)
    return qs.astype(np.float32), qe.astype(np.float32)
