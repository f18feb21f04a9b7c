"""Multi-query probabilistic roadmaps on one GPU, plain and learned-guided.

This is the client side of the collision checker (the reference's planner,
prm/src/lib/prm/prmsolver.cpp, checks every candidate edge eagerly).  Both
planners sample the same seeded configurations, vertex-check them, connect
k nearest free neighbours (L2 in configuration space, like
get_near_vertices, prmsolver.cpp:2533-2574) and answer a batch of
start/goal queries; every collision verdict comes from the exact checker.

* ``plain_prm``: check every candidate edge, take connected components.
* ``lazy_prm``: batched lazy Kruskal, exact connectivity with fewer checks.
    round 1: each vertex's ``first`` lowest-weight candidate edges are
             checked; their free edges define components.
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

The roadmap stays on the device: kNN candidates (gprm_nbr_knn), component
labels, the breadth-first forest the query paths follow and the paths
themselves (gprm_graph_*); the host only sees the final paths.

Time-to-path: wall time from sampling to verified paths for the whole
query batch, divided by the number of queries.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import scenes, workloads
from ._abi import GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT
from .graph import RoadmapGraph
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


def _components(graph, V, i, j, good):
    """Component labels (smallest vertex) of the free-edge graph, on the device."""
    return graph.components(V, i, j, good)


def _answer_queries(cs, graph, verts, i, j, good, label, starts, goals, k):
    """Attaches every start and goal to its k nearest roadmap vertices by
    exactly checked edges, picks the first (start, goal) attachment pair in
    nearest-first order whose vertices share a component, and returns the
    forest paths through the roadmap (all on the device).  Returns
    (paths as host arrays or None, attachment edges checked)."""
    import torch
    dev = verts.device
    Q = starts.shape[0]
    V = verts.shape[0]
    if V == 0:
        return [None] * Q, 0
    ends = torch.cat([torch.as_tensor(starts, device=dev), torch.as_tensor(goals, device=dev)])
    kk = min(k, V)
    index = NeighbourIndex(verts.shape[1])
    index.build(verts.T.contiguous())
    nb = index.knn(kk, q=ends.T.contiguous())[0].long()                       # (2Q, kk)
    qa = ends[:, None, :].expand(-1, kk, -1).reshape(-1, ends.shape[1])
    ok = (_check_edges(cs, qa, verts[nb.reshape(-1)]) == 0).reshape(2 * Q, kk)
    lab = torch.where(ok, label[nb].long(), torch.full_like(nb, -1))
    ls, lg = lab[:Q], lab[Q:]
    match = (ls[:, :, None] == lg[:, None, :]) & (ls[:, :, None] >= 0)       # (Q, kk, kk)
    flat = match.reshape(Q, -1)
    has = flat.any(1)
    first = torch.argmax(flat.to(torch.int8), dim=1)                         # lexicographic first (a, b)
    a, b = first // kk, first % kk
    rows = torch.arange(Q, device=dev)
    vs = torch.where(has, nb[:Q][rows, a], torch.full_like(a, -1)).to(torch.int32)
    vt = torch.where(has, nb[Q:][rows, b], torch.full_like(b, -1)).to(torch.int32)
    parent, depth, _ = graph.forest(V, i, j, label, good)
    length, off, flat_path = graph.paths(vs, vt, label, parent, depth)
    pts = verts[flat_path.long()].cpu().numpy()
    length, off = length.cpu().numpy(), off.cpu().numpy()
    paths = []
    for t in range(Q):
        if length[t] == 0:
            paths.append(None)
            continue
        paths.append(np.concatenate([starts[t:t + 1], pts[off[t]:off[t] + length[t]], goals[t:t + 1]]))
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
    graph = RoadmapGraph()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    q = _sample(scene, n_samples, seed)
    verts = q[_check_vertices(cs, q) == 0]
    i, j = workloads.knn_pairs(verts, k)
    i, j = i.to(torch.int32), j.to(torch.int32)
    good = (_check_edges(cs, verts[i.long()], verts[j.long()]) == 0).to(torch.uint8)
    V = verts.shape[0]
    label = _components(graph, V, i, j, good)
    paths, nconn = _answer_queries(cs, graph, verts, i, j, good, label, starts, goals, k)
    ok = verify_paths(cs, paths)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return PlanResult(np.array([p is not None for p in paths]), paths, dt, int(i.numel()) + nconn,
                      int(cs.stats()["edge_steps_nominal"] - s0), n_samples,
                      {"verified": ok, "free_vertices": V, "candidate_edges": int(i.numel())})


def lazy_prm(cs, scene, starts, goals, n_samples, k=10, seed=0, mlp=None, prune=0.9, beta=4.0,
             batch_frac=1.0, min_batch=4096, max_rounds=2, first=2) -> PlanResult:
    """Batched lazy-Kruskal PRM (exact connectivity), optionally MLP-guided;
    the roadmap and its bookkeeping stay on the device."""
    import torch
    s0 = cs.stats()["edge_steps_nominal"]
    graph = RoadmapGraph()
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
    i64, j64 = workloads.knn_pairs(verts, k)
    i, j = i64.to(torch.int32), j64.to(torch.int32)
    V, E = verts.shape[0], int(i.numel())
    dev = verts.device
    length = torch.linalg.norm(verts[i64] - verts[j64], dim=1)
    if mlp is not None and E:
        pts = torch.cat([verts[i64] + t * (verts[j64] - verts[i64]) for t in (0.25, 0.5, 0.75)])
        pe = mlp.predict(pts.T.contiguous()).reshape(3, -1).max(0).values
        cost = length * (1.0 + beta * pe)
    else:
        cost = length
    good = torch.zeros(E, dtype=torch.uint8, device=dev)
    checked = torch.zeros(E, dtype=torch.bool, device=dev)

    def run(sel):
        if sel.numel() == 0:
            return 0
        ok_ = _check_edges(cs, verts[i64[sel]], verts[j64[sel]]) == 0
        checked[sel] = True
        good[sel] = ok_.to(torch.uint8)
        return int(ok_.sum().item())

    # round 1: every vertex's `first` cheapest candidate edges
    m = int(first)
    ends = torch.cat([i64, j64])
    eid = torch.arange(E, device=dev).repeat(2)
    o = torch.argsort(cost.repeat(2), stable=True)
    o = o[torch.argsort(ends[o], stable=True)]          # by vertex, then cost
    ev = ends[o]
    startpos = torch.searchsorted(ev, torch.arange(V, device=dev))
    rank = torch.arange(2 * E, device=dev) - startpos[ev]
    r1 = torch.unique(eid[o][rank < m])
    free1 = run(r1)
    rounds = [int(r1.numel())]
    order = torch.argsort(cost, stable=True)
    for rnd in range(max_rounds):
        label = _components(graph, V, i, j, good)
        rest = order[~checked[order]]
        cross = rest[label[i64[rest]] != label[j64[rest]]]
        if cross.numel() == 0:
            break
        take = cross if rnd == max_rounds - 1 else cross[:max(min_batch, int(cross.numel() * batch_frac))]
        run(take)
        rounds.append(int(take.numel()))
    label = _components(graph, V, i, j, good)
    paths, nconn = _answer_queries(cs, graph, verts, i, j, good, label, starts, goals, k)
    ok = verify_paths(cs, paths)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return PlanResult(np.array([p is not None for p in paths]), paths, dt, int(checked.sum().item()) + nconn,
                      int(cs.stats()["edge_steps_nominal"] - s0), vchecks,
                      {"verified": ok, "free_vertices": V, "candidate_edges": E, "round1_edges": rounds[0],
                       "round1_free": free1, "later_edges": int(sum(rounds[1:])), "rounds": len(rounds),
                       "pruned": pruned})


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


def predictor_errors(cs, scene, mlp, n=1 << 16, seed=0, prune=0.9):
    """The exact checker as the judge of the predictor on held-out uniform
    configurations: false-free rate (colliding, predicted p < 0.5),
    false-colliding rate (free, predicted p >= 0.5), and the share of free
    configurations the planner would prune (p > prune)."""
    import torch
    q = torch.tensor(np.ascontiguousarray(scenes.uniform_configs(scene, n, seed + 999).T), device="cuda:0")
    codes = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    cs.check_configs_device(q, codes)
    p = mlp.predict(q)
    coll = codes != 0
    free = ~coll
    ncoll, nfree = max(1, int(coll.sum().item())), max(1, int(free.sum().item()))
    return {"held_out": n,
            "false_free_rate": int((coll & (p < 0.5)).sum().item()) / ncoll,
            "false_colliding_rate": int((free & (p >= 0.5)).sum().item()) / nfree,
            "free_pruned_rate": int((free & (p > prune)).sum().item()) / nfree,
            "accuracy": float(((p >= 0.5) == coll).float().mean().item())}


def _summary(r):
    return {"success_rate": float(r.success.mean()), "time_to_path_ms": 1e3 * r.time_to_path,
            "batch_seconds": r.seconds, "edge_checks": r.edge_checks, "edge_steps": r.edge_steps,
            "vertex_checks": r.vertex_checks, "paths_verified": bool(r.info["verified"]),
            **{k_: (v.item() if isinstance(v, np.generic) else v) for k_, v in r.info.items() if k_ != "verified"}}


def _median_run(fn, repeats):
    fn()
    rs = [fn() for _ in range(repeats)]
    return sorted(rs, key=lambda x: x.seconds)[len(rs) // 2]


def compare_planners(cs, scene, n_samples=1 << 16, n_queries=1000, k=10, seed=0, mlp=None, repeats=3,
                     first=2, max_rounds=2):
    """Plain (eager) PRM against the lazy PRM without guidance and the
    learned-guided lazy PRM, on the same seeded queries.  Each run is
    repeated (`repeats` timed runs after one untimed) and the median is
    reported.  The lazy PRM has the eager PRM's connectivity on the same
    samples, so its success rate is the same by construction.  The learned
    PRM prunes samples, which can change the roadmap: it runs on
    n_samples, then on 1.125x, 1.25x, ... samples until its success rate
    reaches the plain planner's, and the time of that run is the one
    compared ("equal success rate")."""
    starts, goals = make_queries(cs, scene, n_queries, seed + 17)
    out = {}
    plain = _median_run(lambda: plain_prm(cs, scene, starts, goals, n_samples, k, seed), repeats)
    out["plain"] = _summary(plain)
    lazy = _median_run(lambda: lazy_prm(cs, scene, starts, goals, n_samples, k, seed, first=first,
                                        max_rounds=max_rounds), repeats)
    out["lazy"] = _summary(lazy)
    if mlp is not None:
        target = float(plain.success.mean())
        n, tries = n_samples, []
        for _ in range(8):
            r = _median_run(lambda: lazy_prm(cs, scene, starts, goals, n, k, seed, mlp=mlp, first=first,
                                             max_rounds=max_rounds), repeats)
            tries.append({"samples": n, "success_rate": float(r.success.mean()), "time_to_path_ms": 1e3 * r.time_to_path})
            if r.success.mean() >= target:
                break
            n = int(n * 1.125)
        out["learned"] = dict(_summary(r), samples=n, sample_search=tries,
                              success_matched=bool(r.success.mean() >= target))
        out["learned_over_plain_time"] = out["learned"]["time_to_path_ms"] / out["plain"]["time_to_path_ms"]
        out["learned_over_lazy_time"] = out["learned"]["time_to_path_ms"] / out["lazy"]["time_to_path_ms"]
        out["predictor_errors"] = predictor_errors(cs, scene, mlp, seed=seed)
    out["lazy_over_plain_time"] = out["lazy"]["time_to_path_ms"] / out["plain"]["time_to_path_ms"]
    out["config"] = {"samples": n_samples, "queries": n_queries, "k": k, "seed": seed, "dq": float(cs.deltaq()),
                     "lazy_first": first, "lazy_rounds": max_rounds}
    return out
