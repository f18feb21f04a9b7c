"""Roadmap graph operations: the Dijkstra restatement pinned against the
reference's own do_dijkstra (prmsolver.cpp:2805-2846, compiled from its
sources into oracle/_ref/libnbr_ref.so), and the device kernels checked
against the restatements exactly (labels, parents, depths, paths,
float32 distances)."""
import ctypes as C
import os

import numpy as np
import pytest

import graph_oracle as GO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnbr_ref.so")


def _geometric_graph(n, ndof, radius, seed, drop=0.0):
    """Nodes uniform in [-pi, pi]^ndof, edges between nodes closer than
    radius (weights = float32 distances), a fraction `drop` removed."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-np.pi, np.pi, (n, ndof)).astype(np.float32)
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    eu, ev = np.nonzero(np.triu(d2 < radius * radius, 1))
    keep = rng.random(len(eu)) >= drop
    eu, ev = eu[keep].astype(np.int32), ev[keep].astype(np.int32)
    w = np.sqrt(((x[eu] - x[ev]) ** 2).sum(-1)).astype(np.float32)
    return x, eu, ev, w


def test_oracle_forest_paths_are_valid():
    x, eu, ev, _ = _geometric_graph(300, 3, 1.2, 1)
    lab = GO.components(300, eu, ev)
    parent, depth = GO.forest(300, eu, ev, lab)
    edges = set(zip(eu.tolist(), ev.tolist())) | set(zip(ev.tolist(), eu.tolist()))
    for s, t in [(0, 1), (5, 77), (100, 250)]:
        if lab[s] != lab[t]:
            continue
        p = GO.forest_path(parent, depth, s, t)
        assert p[0] == s and p[-1] == t
        assert all((a, b) in edges for a, b in zip(p[:-1], p[1:]))


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref/libnbr_ref.so not built")
@pytest.mark.parametrize("ndof,n,radius,seed", [(4, 400, 1.3, 2), (6, 500, 2.2, 3)])
def test_oracle_dijkstra_matches_reference(ndof, n, radius, seed):
    lib = C.CDLL(REF_LIB)
    x, eu, ev, w = _geometric_graph(n, ndof, radius, seed)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    lab = GO.components(n, eu, ev)
    rng = np.random.default_rng(seed)
    tried = 0
    for _ in range(40):
        s, t = (int(v) for v in rng.integers(0, n, 2))
        if s == t or lab[s] != lab[t]:
            continue
        path = np.zeros(n, np.int32)
        dto = C.c_float(0)
        L = lib.ref_dijkstra(ndof, P(x), n, P(eu), P(ev), P(w), len(eu), s, t, P(path), n, C.byref(dto))
        assert L > 0
        dist, parent = GO.dijkstra(n, eu, ev, w, s)
        assert np.float32(dto.value) == dist[t]
        ref_path = path[:L][::-1]          # the reference lists goal first
        # the reference path is a shortest path under the same float sums
        acc = np.float32(0)
        wmap = {(int(a), int(b)): wv for a, b, wv in zip(eu, ev, w)}
        for a, b in zip(ref_path[:-1], ref_path[1:]):
            acc = np.float32(acc + wmap.get((int(a), int(b)), wmap.get((int(b), int(a)))))
        assert acc == dist[t]
        # and, away from exact ties, the same path as the smallest-parent rule
        mine = [t]
        while mine[-1] != s:
            mine.append(int(parent[mine[-1]]))
        if len(mine) == L:
            np.testing.assert_array_equal(np.array(mine[::-1]), ref_path)
        tried += 1
    assert tried >= 10


@pytest.mark.gpu
@pytest.mark.parametrize("n,ndof,radius,drop", [(2000, 3, 0.9, 0.0), (5000, 4, 1.1, 0.3), (300, 2, 0.2, 0.0)])
def test_gpu_components_forest_paths(n, ndof, radius, drop):
    import torch
    from gpuprm_b200.graph import RoadmapGraph
    x, eu, ev, w = _geometric_graph(n, ndof, radius, 11, drop)
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(12)
    mask = (rng.random(len(eu)) < 0.9).astype(np.uint8)
    G = RoadmapGraph()
    teu, tev = torch.tensor(eu, device=dev), torch.tensor(ev, device=dev)
    tm = torch.tensor(mask, device=dev)
    lab = G.components(n, teu, tev, tm)
    want = GO.components(n, eu[mask == 1], ev[mask == 1])
    np.testing.assert_array_equal(lab.cpu().numpy(), want)
    parent, depth, levels = G.forest(n, teu, tev, lab, tm)
    wp, wd = GO.forest(n, eu[mask == 1], ev[mask == 1], want)
    INF = np.iinfo(np.int32).max
    np.testing.assert_array_equal(parent.cpu().numpy(), wp)
    np.testing.assert_array_equal(depth.cpu().numpy(), np.where(wd == INF, INF, wd))
    qs = rng.integers(0, n, 300).astype(np.int32)
    qt = rng.integers(0, n, 300).astype(np.int32)
    length, off, flat = G.paths(torch.tensor(qs, device=dev), torch.tensor(qt, device=dev), lab, parent, depth)
    length, off, flat = length.cpu().numpy(), off.cpu().numpy(), flat.cpu().numpy()
    for t in range(300):
        if want[qs[t]] != want[qt[t]]:
            assert length[t] == 0
            continue
        np.testing.assert_array_equal(flat[off[t]:off[t] + length[t]],
                                      GO.forest_path(wp, wd, int(qs[t]), int(qt[t])))


@pytest.mark.gpu
@pytest.mark.parametrize("n,ndof,radius", [(1500, 3, 0.8), (3000, 4, 1.2)])
def test_gpu_sssp_matches_dijkstra(n, ndof, radius):
    import torch
    from gpuprm_b200.graph import RoadmapGraph
    x, eu, ev, w = _geometric_graph(n, ndof, radius, 21)
    dev = torch.device("cuda:0")
    G = RoadmapGraph()
    for src in (0, n // 2, n - 1):
        dist, parent, _ = G.sssp(n, torch.tensor(eu, device=dev), torch.tensor(ev, device=dev),
                                 torch.tensor(w, device=dev), src)
        wd, wp = GO.dijkstra(n, eu, ev, w, src)
        np.testing.assert_array_equal(dist.cpu().numpy(), wd)
        np.testing.assert_array_equal(parent.cpu().numpy(), wp)
