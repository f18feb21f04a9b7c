"""Multi-query probabilistic roadmaps on one GPU, plain and learned-guided.

This is the client side of the collision checker (the reference's planner,
prm/src/lib/prm/prmsolver.cpp, checks every candidate edge eagerly).  Both
planners sample the same seeded configurations, vertex-check them, connect
k nearest free neighbours (L2 in configuration space, like
get_near_vertices, prmsolver.cpp:2533-2574) and answer a batch of
start/goal queries; every collision verdict comes from the exact checker.

* ``plain_prm``: check every candidate edge, take connected components.
* ``lazy_prm``: batched lazy Kruskal, exact connectivity with fewer checks.
    round 1: each vertex's ``first`` lowest-weight candidate edges (or,
             with first="mst", a minimum spanning forest) are checked; their
             free edges define components.
    round r: the unchecked edges that join two different components, in
             weight order, are checked in one batch (the first
             ``batch_frac`` of them, all of them in the last round); the
             components are recomputed.
  It stops when no unchecked edge joins two components.  Every free
  candidate edge is then either checked or inside a component, so the
  components are exactly those of the fully checked graph: the same
  queries succeed.  With a trained ``CollisionMLP`` the samples with
  predicted P(collision) > ``prune`` are dropped before the vertex check
  and edges are weighted by length * (1 + beta * p_edge) (p_edge: largest
  prediction at three interior points), so likely-free edges are checked
  first and likely-colliding ones tend to become internal before their
  turn.  Without one, edges are weighted by length.
* Every returned path is re-checked edge by edge with the all-steps policy
  (``verify_paths``).

Time-to-path: wall time from sampling to verified paths for the whole
query batch, divided by the number of queries.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import scenes, workloads
from ._abi import GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT
from .neighbours import NeighbourIndex


@dataclass
class PlanResult:
    success: np.ndarray            # (Q,) bool
    paths: list                    # list of (L, ndof) arrays or None
    seconds: float                 # wall time for the whole query batch
    edge_checks: int               # edges sent to the exact checker
    edge_steps: int                # nominal edge steps checked
    vertex_checks: int
    info: dict = field(default_factory=dict)

    @property
    def time_to_path(self) -> float:
        return self.seconds / max(1, len(self.success))


def _check_edges(cs, qa, qb, policy=GPRM_EDGES_EARLY_EXIT):
    """Exact verdicts (int32 codes) of edges qa[i] -> qb[i] ((n, ndof) CUDA tensors)."""
    import torch
    n = qa.shape[0]
    if n == 0:
        return torch.zeros(0, dtype=torch.int32, device=qa.device)
    cs.set_edge_policy(policy)
    res = torch.empty(n, dtype=torch.int32, device=qa.device)
    cs.check_edges_device(qa.T.contiguous(), qb.T.contiguous(), res)
    return res


def _check_vertices(cs, q):
    import torch
    res = torch.empty(q.shape[0], dtype=torch.int32, device=q.device)
    if q.shape[0]:
        cs.check_configs_device(q.T.contiguous(), res)
    return res


def _components(V, ei, ej):
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    return connected_components(coo_matrix((np.ones(len(ei)), (ei, ej)), shape=(V, V)), directed=False)[1]


def _bfs_parents(V, ei, ej, comp):
    """Parent pointers of a BFS forest of the graph (ei, ej), one root per
    component (its smallest vertex); level-synchronous, vectorised."""
    from scipy.sparse import coo_matrix
    A = coo_matrix((np.ones(len(ei), np.int8), (ei, ej)), shape=(V, V)).tocsr()
    A = (A + A.T).tocsr()
    parent = np.full(V, -2, np.int64)
    _, roots = np.unique(comp, return_index=True)
    parent[roots] = -1
    frontier = roots
    while len(frontier):
        starts = A.indptr[frontier]
        cnt = A.indptr[frontier + 1] - starts
        src = np.repeat(frontier, cnt)
        idx = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt) + np.repeat(starts, cnt)
        nb = A.indices[idx]
        new = parent[nb] == -2
        nb, src = nb[new], src[new]
        nb, first = np.unique(nb, return_index=True)
        parent[nb] = src[first]
        frontier = nb
    return parent


def _tree_path(parent, s, t):
    a, b = [s], [t]
    seen = {s: 0}
    while parent[a[-1]] >= 0:
        a.append(int(parent[a[-1]]))
        seen[a[-1]] = len(a) - 1
    while b[-1] not in seen:
        if parent[b[-1]] < 0:
            return None
        b.append(int(parent[b[-1]]))
    return a[:seen[b[-1]]] + b[::-1]


def _answer_queries(cs, verts, comp, parent, starts, goals, k):
    """Attaches starts and goals to up to k nearest roadmap vertices with
    exactly checked edges and returns the paths through the BFS forest."""
    import torch
    Q = starts.shape[0]
    st = torch.as_tensor(starts, device=verts.device)
    gl = torch.as_tensor(goals, device=verts.device)
    ends = torch.cat([st, gl])
    kk = min(k, verts.shape[0])
    index = NeighbourIndex(verts.shape[1])
    index.build(verts.T.contiguous())
    nb = index.knn(kk, q=ends.T.contiguous())[0].long()
    qa = ends[:, None, :].expand(-1, kk, -1).reshape(-1, ends.shape[1])
    res = _check_edges(cs, qa, verts[nb.reshape(-1)]).reshape(2 * Q, kk)
    ok = (res == 0).cpu().numpy()
    nbn = nb.cpu().numpy()
    c = np.where(ok, comp[nbn], -1)
    cs_, cg_ = c[:Q], c[Q:]
    # first start attachment whose component some goal attachment shares
    match = (cs_[:, :, None] == cg_[:, None, :]) & (cs_[:, :, None] >= 0)
    has = match.any(axis=(1, 2))
    verts_np = verts.cpu().numpy()
    paths = []
    for i in range(Q):
        if not has[i]:
            paths.append(None)
            continue
        a, b = np.argwhere(match[i])[0]
        p = _tree_path(parent, int(nbn[i, a]), int(nbn[Q + i, b]))
        if p is None:
            paths.append(None)
            continue
        paths.append(np.concatenate([starts[i:i + 1], verts_np[p], goals[i:i + 1]]))
    return paths, 2 * Q * kk


def verify_paths(cs, paths):
    """Re-checks every edge of every path (all-steps policy); True if all free."""
    import torch
    segs_a = [p[:-1] for p in paths if p is not None and len(p) > 1]
    segs_b = [p[1:] for p in paths if p is not None and len(p) > 1]
    if not segs_a:
        return True
    seg = np.unique(np.concatenate([np.concatenate(segs_a), np.concatenate(segs_b)], axis=1), axis=0)
    d = seg.shape[1] // 2
    qa = torch.tensor(seg[:, :d], device="cuda:0", dtype=torch.float32)
    qb = torch.tensor(seg[:, d:], device="cuda:0", dtype=torch.float32)
    return bool((_check_edges(cs, qa, qb, GPRM_EDGES_ALL_STEPS) == 0).all().item())


def _sample(scene, n, seed):
    """n configurations uniform in the joint box, drawn on the GPU (seeded)."""
    import torch
    g = torch.Generator(device="cuda:0")
    g.manual_seed(seed)
    lo = torch.tensor(scene.mins, device="cuda:0")
    hi = torch.tensor(scene.maxs, device="cuda:0")
    return lo + (hi - lo) * torch.rand((n, scene.ndof), device="cuda:0", generator=g)


def plain_prm(cs, scene, starts, goals, n_samples, k=10, seed=0) -> PlanResult:
    """Eager GPU PRM: every vertex and every candidate edge checked."""
    import torch
    s0 = cs.stats()["edge_steps_nominal"]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    q = _sample(scene, n_samples, seed)
    verts = q[_check_vertices(cs, q) == 0]
    i, j = workloads.knn_pairs(verts, k)
    good = (_check_edges(cs, verts[i], verts[j]) == 0).cpu().numpy()
    ei, ej = i.cpu().numpy()[good], j.cpu().numpy()[good]
    V = verts.shape[0]
    comp = _components(V, ei, ej)
    parent = _bfs_parents(V, ei, ej, comp)
    paths, nconn = _answer_queries(cs, verts, comp, parent, starts, goals, k)
    ok = verify_paths(cs, paths)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return PlanResult(np.array([p is not None for p in paths]), paths, dt, int(len(good)) + nconn,
                      int(cs.stats()["edge_steps_nominal"] - s0), n_samples,
                      {"verified": ok, "free_vertices": V, "candidate_edges": int(len(good))})


def lazy_prm(cs, scene, starts, goals, n_samples, k=10, seed=0, mlp=None, prune=0.9, beta=4.0,
             batch_frac=1.0, min_batch=4096, max_rounds=2, first=2) -> PlanResult:
    """Batched lazy-Kruskal PRM (exact connectivity), optionally MLP-guided."""
    import torch
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import minimum_spanning_tree
    s0 = cs.stats()["edge_steps_nominal"]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    q = _sample(scene, n_samples, seed)
    pruned = 0
    if mlp is not None:
        keep = mlp.predict(q.T.contiguous()) <= prune
        pruned = int((~keep).sum().item())
        q = q[keep]
    verts = q[_check_vertices(cs, q) == 0]
    vchecks = int(q.shape[0])
    i, j = workloads.knn_pairs(verts, k)
    V, E = verts.shape[0], int(i.shape[0])
    length = torch.linalg.norm(verts[i] - verts[j], dim=1)
    if mlp is not None:
        pts = torch.cat([verts[i] + t * (verts[j] - verts[i]) for t in (0.25, 0.5, 0.75)])
        pe = mlp.predict(pts.T.contiguous()).reshape(3, -1).max(0).values
        cost = length * (1.0 + beta * pe)
    else:
        cost = length
    ii, jj = i.cpu().numpy(), j.cpu().numpy()
    w = cost.cpu().numpy().astype(np.float64) + 1e-9
    good = np.zeros(E, bool)
    checked = np.zeros(E, bool)

    def run(sel):
        t = torch.as_tensor(sel, device="cuda:0")
        ok_ = (_check_edges(cs, verts[i[t]], verts[j[t]]) == 0).cpu().numpy()
        checked[sel] = True
        good[sel[ok_]] = True
        return int(ok_.sum())

    if first == "mst":
        # round 1: the minimum spanning forest
        T = minimum_spanning_tree(coo_matrix((w, (ii, jj)), shape=(V, V))).tocoo()
        key = ii.astype(np.int64) * V + jj
        korder = np.argsort(key)
        tk = np.minimum(T.row, T.col).astype(np.int64) * V + np.maximum(T.row, T.col)
        r1 = korder[np.searchsorted(key[korder], tk)]
    else:
        # round 1: every vertex's `first` cheapest candidate edges (on the GPU)
        m = int(first)
        ends = torch.cat([i, j])
        eid = torch.arange(E, device="cuda:0").repeat(2)
        c2 = cost.repeat(2)
        o = torch.argsort(c2, stable=True)
        o = o[torch.argsort(ends[o], stable=True)]          # by vertex, then cost
        ev = ends[o]
        startpos = torch.searchsorted(ev, torch.arange(V, device="cuda:0"))
        rank = torch.arange(2 * E, device="cuda:0") - startpos[ev]
        r1 = torch.unique(eid[o][rank < m]).cpu().numpy()
    free1 = run(r1)
    rounds = [len(r1)]
    order = np.argsort(w, kind="stable")
    for rnd in range(max_rounds):
        comp_r = _components(V, ii[good], jj[good])
        rest = order[~checked[order]]
        cross = rest[comp_r[ii[rest]] != comp_r[jj[rest]]]
        if len(cross) == 0:
            break
        take = cross if rnd == max_rounds - 1 else cross[:max(min_batch, int(len(cross) * batch_frac))]
        run(take)
        rounds.append(len(take))
    r2n = int(sum(rounds[1:]))
    ei, ej = ii[good], jj[good]
    comp = _components(V, ei, ej)
    parent = _bfs_parents(V, ei, ej, comp)
    paths, nconn = _answer_queries(cs, verts, comp, parent, starts, goals, k)
    ok = verify_paths(cs, paths)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return PlanResult(np.array([p is not None for p in paths]), paths, dt, int(checked.sum()) + nconn,
                      int(cs.stats()["edge_steps_nominal"] - s0), vchecks,
                      {"verified": ok, "free_vertices": V, "candidate_edges": E, "round1_edges": int(len(r1)),
                       "round1_free": free1, "later_edges": r2n, "rounds": len(rounds), "pruned": pruned})


def make_queries(cs, scene, n_queries, seed):
    """Seeded start/goal pairs among exactly checked free configurations."""
    need = 2 * n_queries
    got, s = [], 0
    while sum(len(g) for g in got) < need:
        q = scenes.uniform_configs(scene, 4 * need, seed + 424242 + s)
        got.append(q[cs.check_configs(q) == 0])
        s += 1
    allq = np.concatenate(got)[:need]
    return allq[:n_queries].copy(), allq[n_queries:].copy()


def train_predictor(cs, scene, n_labels=1 << 20, epochs=10, batch=4096, lr=1e-3, seed=0):
    """Trains a CollisionMLP on exact-checker labels of uniform samples.
    Returns (mlp, per-epoch losses, seconds of label generation, seconds of training)."""
    import torch
    from .mlp import CollisionMLP
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    q = torch.tensor(np.ascontiguousarray(scenes.uniform_configs(scene, n_labels, seed + 101).T), device="cuda:0")
    codes = torch.zeros(n_labels, dtype=torch.int32, device="cuda:0")
    cs.check_configs_device(q, codes)
    y = (codes != 0).float()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    mlp = CollisionMLP(scene.ndof, seed=seed)
    losses = mlp.train(q, y, epochs=epochs, batch=batch, lr=lr, seed=seed + 1)
    torch.cuda.synchronize()
    return mlp, losses, t1 - t0, time.perf_counter() - t1


def compare_planners(cs, scene, n_samples=1 << 16, n_queries=1000, k=10, seed=0, mlp=None, repeats=3):
    """Plain (eager) PRM against the learned-guided lazy PRM (and the lazy PRM
    without guidance) on the same seeded samples and queries.  Each method
    runs once untimed, then `repeats` times; the median is reported."""
    starts, goals = make_queries(cs, scene, n_queries, seed + 17)
    out = {}
    runs = {"plain": lambda: plain_prm(cs, scene, starts, goals, n_samples, k, seed),
            "lazy": lambda: lazy_prm(cs, scene, starts, goals, n_samples, k, seed),
            "learned": lambda: lazy_prm(cs, scene, starts, goals, n_samples, k, seed, mlp=mlp)}
    for name, fn in runs.items():
        if name == "learned" and mlp is None:
            continue
        fn()
        rs = [fn() for _ in range(repeats)]
        r = sorted(rs, key=lambda x: x.seconds)[len(rs) // 2]
        out[name] = {"success_rate": float(r.success.mean()), "time_to_path_ms": 1e3 * r.time_to_path,
                     "batch_seconds": r.seconds, "edge_checks": r.edge_checks, "edge_steps": r.edge_steps,
                     "vertex_checks": r.vertex_checks, "paths_verified": bool(r.info["verified"]),
                     **{k_: (v.item() if isinstance(v, np.generic) else v) for k_, v in r.info.items()
                        if k_ != "verified"}}
    if "learned" in out:
        out["learned_over_plain_time"] = out["learned"]["time_to_path_ms"] / out["plain"]["time_to_path_ms"]
    out["config"] = {"samples": n_samples, "queries": n_queries, "k": k, "seed": seed}
    return out
