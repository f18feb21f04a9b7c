"""Roadmap output in the reference planner's result format.

GPUPRM stores a finished run with PRMSolver::store_results / store_graph
(prm/src/lib/prm/prmsolver.cpp:2947-3055) for its MATLAB plotting scripts:

    <path>/connection.bin          start and goal connected (first byte)
    <path>/graphl/, graphr/        one directory per roadmap:
        qstorage.bin   float  node storage, ndof per position (unused = 0)
        surrnum.bin    int    neighbour count per position
        edgesfrom.bin, edgesto.bin   int  edge endpoints (positions)
        edgesweight.bin              int  edge length, truncated to int
        edgesfromc.bin, edgestoc.bin int  the same in compressed numbering
        qstoragec.bin  float  the used positions only, in block order
        blockpos.bin   int    first position of each block
        blocknum.bin   int    the number of blocks (written last, over the
                              per-block counts the reference writes first)
        newblockpos.bin, numc.bin, startc.bin, endc.bin   int
        path.bin, pathc.bin  int  the Dijkstra path, goal first (only when
                              start and goal are connected)

A roadmap is given as its block layout (``Roadmap``): the reference stores
nodes in blocks of ``blocksize`` positions keyed by the first joint;
edges are per-position adjacency lists with float weights.  ``Roadmap.from_edges``
builds one from a flat vertex array (consecutive blocks, no gaps), so the
device planners can write their roadmaps in this format.
"""
from __future__ import annotations

import os
import shutil
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Roadmap:
    ndof: int
    qstorage: np.ndarray            # (newblockpos * ndof,) float32
    surrnum: np.ndarray             # (newblockpos,) int32
    blocks: np.ndarray              # (blocknum, 2) int32: (pos, num)
    adj_off: np.ndarray             # (newblockpos + 1,) CSR offsets over positions
    adj_dest: np.ndarray            # int32 neighbour positions
    adj_w: np.ndarray               # float32 weights
    start: int                      # position of the path's start
    end: int                        # position of the path's end
    path: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))   # positions, goal first

    @property
    def newblockpos(self) -> int:
        return int(self.surrnum.shape[0])

    @staticmethod
    def from_edges(q, ei, ej, start: int, end: int, path=None, blocksize: int = 256) -> "Roadmap":
        """Roadmap of vertices q (n, ndof) and undirected edges (ei[e], ej[e]),
        weights = float32 Euclidean length, stored in consecutive blocks of
        `blocksize` positions.  `path` lists vertex ids from start to end."""
        q = np.ascontiguousarray(q, np.float32)
        n, ndof = q.shape
        ei = np.asarray(ei, np.int64)
        ej = np.asarray(ej, np.int64)
        nb = max(1, (n + blocksize - 1) // blocksize)
        newblockpos = nb * blocksize
        qs = np.zeros(newblockpos * ndof, np.float32)
        qs[:n * ndof] = q.reshape(-1)
        w = np.sqrt(((q[ei] - q[ej]) ** 2).sum(1, dtype=np.float32)).astype(np.float32)
        src = np.concatenate([ei, ej])
        dst = np.concatenate([ej, ei])
        ww = np.concatenate([w, w])
        order = np.argsort(src, kind="stable")
        src, dst, ww = src[order], dst[order], ww[order]
        cnt = np.bincount(src, minlength=newblockpos)
        off = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int32)
        blocks = np.array([(b * blocksize, min(blocksize, n - b * blocksize)) for b in range(nb)], np.int32)
        p = np.zeros(0, np.int32) if path is None else np.asarray(path, np.int32)[::-1].copy()
        return Roadmap(ndof, qs, cnt.astype(np.int32), blocks, off, dst.astype(np.int32), ww, int(start), int(end), p)


def _w(path: str, arr, dtype) -> None:
    np.ascontiguousarray(arr, dtype).tofile(path)


def store_graph(path: str, g: Roadmap) -> None:
    """store_graph(path, g, d, start, end) (prmsolver.cpp:2981-3055)."""
    os.makedirs(path, exist_ok=True)
    n = g.newblockpos
    _w(os.path.join(path, "qstorage.bin"), g.qstorage[:g.ndof * n], np.float32)
    _w(os.path.join(path, "surrnum.bin"), g.surrnum[:n], np.int32)
    posmapping = np.zeros(max(n, 1), np.int64)
    ef, et, ew, qc, bpos, bnum = [], [], [], [], [], []
    index = 0
    for pos0, num in g.blocks:
        bpos.append(pos0)
        bnum.append(num)
        for l in range(pos0, pos0 + num):
            qc.append(g.qstorage[g.ndof * l:g.ndof * (l + 1)])
            posmapping[l] = index
            a, b = g.adj_off[l], g.adj_off[l + 1]
            ef.append(np.full(b - a, l, np.int32))
            et.append(g.adj_dest[a:b])
            ew.append(g.adj_w[a:b])
            index += 1
    cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt)
    ef, et = cat(ef, np.int32), cat(et, np.int32)
    ew = np.trunc(cat(ew, np.float32)).astype(np.int32)         # int(weight) as in a float -> int push_back
    _w(os.path.join(path, "edgesfrom.bin"), ef, np.int32)
    _w(os.path.join(path, "edgesto.bin"), et, np.int32)
    _w(os.path.join(path, "edgesfromc.bin"), posmapping[ef], np.int32)
    _w(os.path.join(path, "edgestoc.bin"), posmapping[et], np.int32)
    _w(os.path.join(path, "edgesweight.bin"), ew, np.int32)
    _w(os.path.join(path, "qstoragec.bin"), cat(qc, np.float32), np.float32)
    _w(os.path.join(path, "blockpos.bin"), np.array(bpos, np.int32), np.int32)
    _w(os.path.join(path, "blocknum.bin"), np.array(bnum, np.int32), np.int32)
    _w(os.path.join(path, "newblockpos.bin"), [n], np.int32)
    _w(os.path.join(path, "blocknum.bin"), [len(g.blocks)], np.int32)     # overwrites the counts, as the reference does
    _w(os.path.join(path, "numc.bin"), [index], np.int32)
    _w(os.path.join(path, "startc.bin"), [posmapping[g.start]], np.int32)
    _w(os.path.join(path, "endc.bin"), [posmapping[g.end]], np.int32)
    if len(g.path):
        _w(os.path.join(path, "path.bin"), g.path, np.int32)
        _w(os.path.join(path, "pathc.bin"), posmapping[g.path], np.int32)


def store_results(path: str, graphl: Roadmap, graphr: Roadmap, connected: bool) -> None:
    """store_results(path) (prmsolver.cpp:2947-2979): replaces `path`."""
    if os.path.isdir(path):
        shutil.rmtree(path)
    os.makedirs(path)
    store_graph(os.path.join(path, "graphl"), graphl if connected else _no_path(graphl))
    store_graph(os.path.join(path, "graphr"), graphr if connected else _no_path(graphr))
    _w(os.path.join(path, "connection.bin"), [1 if connected else 0], np.int32)


def _no_path(g: Roadmap) -> Roadmap:
    return Roadmap(g.ndof, g.qstorage, g.surrnum, g.blocks, g.adj_off, g.adj_dest, g.adj_w, g.start, g.end,
                   np.zeros(0, np.int32))


def load_graph(path: str, ndof: int) -> dict:
    """Reads one graph directory written by store_graph (as the MATLAB
    scripts do): every array by name."""
    r = lambda name, dt: np.fromfile(os.path.join(path, name), dt) if os.path.exists(os.path.join(path, name)) else None
    out = {name[:-4]: r(name, dt) for name, dt in (
        ("qstorage.bin", np.float32), ("surrnum.bin", np.int32), ("edgesfrom.bin", np.int32),
        ("edgesto.bin", np.int32), ("edgesfromc.bin", np.int32), ("edgestoc.bin", np.int32),
        ("edgesweight.bin", np.int32), ("qstoragec.bin", np.float32), ("blockpos.bin", np.int32),
        ("blocknum.bin", np.int32), ("newblockpos.bin", np.int32), ("numc.bin", np.int32),
        ("startc.bin", np.int32), ("endc.bin", np.int32), ("path.bin", np.int32), ("pathc.bin", np.int32))}
    out["qstorage"] = out["qstorage"].reshape(-1, ndof)
    out["qstoragec"] = out["qstoragec"].reshape(-1, ndof)
    return out


def load_dump(path: str) -> Roadmap:
    """A roadmap from the raw arrays the reference-planner harness dumps."""
    r = lambda name, dt: np.fromfile(os.path.join(path, name), dt)
    ndof, blocknum, n, start, end, plen = (int(v) for v in r("meta.bin", np.int32))
    path_ = r("path.bin", np.int32) if plen and os.path.exists(os.path.join(path, "path.bin")) else np.zeros(0, np.int32)
    return Roadmap(ndof, r("qstorage.bin", np.float32), r("surrnum.bin", np.int32),
                   r("blocks.bin", np.int32).reshape(-1, 2), r("adj_off.bin", np.int32), r("adj_dest.bin", np.int32),
                   r("adj_w.bin", np.float32), start, end, path_)


def store_plan(path: str, result, verts, ei, ej, query: int = 0) -> None:
    """Writes a device planner's roadmap for one query in this format: the
    roadmap (free vertices and free edges) as graphl with the query's start
    attached and its path, and the goal alone as graphr; connected when the
    query was solved.  `result` is a planner.PlanResult, verts (n, ndof),
    (ei, ej) the free roadmap edges."""
    verts = np.asarray(verts, np.float32)
    n = verts.shape[0]
    dp = result.device_paths
    p = result.paths[query]
    st, gl = np.asarray(dp.starts[query], np.float32), np.asarray(dp.goals[query], np.float32)
    q = np.concatenate([verts, st[None], gl[None]])
    s_id, g_id = n, n + 1
    ei, ej = list(np.asarray(ei)), list(np.asarray(ej))
    path_ids = None
    if p is not None:
        length, off, flat = (x.cpu().numpy() for x in (dp.length, dp.off, dp.flat))
        mid = flat[off[query]:off[query] + length[query]].tolist()
        path_ids = [s_id] + mid + [g_id]
        ei += [s_id, mid[-1]]
        ej += [mid[0], g_id]
    gl_map = Roadmap.from_edges(q, ei, ej, start=s_id, end=g_id if p is not None else s_id, path=path_ids)
    gr_map = Roadmap.from_edges(gl[None], [], [], start=0, end=0)
    store_results(path, gl_map, gr_map, p is not None)
