"""Multi-query probabilistic roadmaps on one GPU, plain and learned-guided.

This is the client side of the collision checker (the reference's planner,
prm/src/lib/prm/prmsolver.cpp, checks every candidate edge eagerly).  Both
planners sample the same seeded configurations, vertex-check them, connect
k nearest free neighbours (L2 in configuration space, like
get_near_vertices, prmsolver.cpp:2533-2574) and answer a batch of
start/goal queries; every collision verdict comes from the exact checker.

* ``plain_prm``: check every candidate edge, take connected components.
* ``lazy_prm``: batched lazy Boruvka, exact connectivity with fewer checks.
    round 1: each vertex's ``first`` lowest-weight candidate edges are
             checked; their free edges define components.
    round r: each component's m lowest-weight unchecked edges to other
             components are checked in one batch (m = first * growth^(r-1));
             the last round (``max_rounds``) checks every such edge; the
             components are recomputed after each round.
  It stops when no unchecked edge joins two components.  Every free
  candidate edge is then either checked or inside a component, so the
  components are exactly those of the fully checked graph: the same
  queries succeed.  With a trained ``CollisionMLP`` the samples with
  predicted P(collision) > ``prune`` are dropped before the vertex check
  and edges are weighted by length * (1 + beta * p_edge) (p_edge: the
  prediction at the edge's midpoint), so likely-free edges are checked
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

from . import scenes
from ._abi import GPRM_EDGES_ALL_STEPS
from .graph import RoadmapGraph
from .neighbours import NeighbourIndex


class DevicePaths:
    """The planner's answer kept on the device: for query t, the path is
    start[t], verts[flat[off[t] : off[t] + length[t]]], goal[t] (length 0:
    no path).  Host arrays are built on first access."""

    def __init__(self, verts, length, off, flat, starts, goals):
        self.verts, self.length, self.off, self.flat = verts, length, off, flat
        self.starts, self.goals = starts, goals
        self._host = None

    def __len__(self):
        return int(self.length.numel())

    def found(self) -> np.ndarray:
        return (self.length > 0).cpu().numpy()

    def to_list(self):
        if self._host is None:
            pts = self.verts[self.flat.long()].cpu().numpy()
            length, off = self.length.cpu().numpy(), self.off.cpu().numpy()
            out = []
            for t in range(len(length)):
                if length[t] == 0:
                    out.append(None)
                    continue
                out.append(np.concatenate([self.starts[t:t + 1], pts[off[t]:off[t] + length[t]],
                                           self.goals[t:t + 1]]))
            self._host = out
        return self._host


@dataclass
class PlanResult:
    success: np.ndarray            # (Q,) bool
    device_paths: DevicePaths      # paths on the device
    seconds: float                 # wall time for the whole query batch
    edge_checks: int               # edges sent to the exact checker
    edge_steps: int                # nominal edge steps checked
    vertex_checks: int
    info: dict = field(default_factory=dict)

    @property
    def paths(self):
        """list of (L, ndof) arrays (start ... goal) or None per query."""
        return self.device_paths.to_list()

    @property
    def time_to_path(self) -> float:
        return self.seconds / max(1, len(self.success))


class _Phases:
    """Wall time per planner phase (synchronising at each mark) when enabled."""

    def __init__(self, on: bool):
        self.on = on
        self.t = {}
        self.last = None

    def mark(self, name):
        if not self.on:
            return
        import torch
        torch.cuda.synchronize()
        now = time.perf_counter()
        if self.last is not None:
            self.t[name] = self.t.get(name, 0.0) + 1e3 * (now - self.last)
        self.last = now


def _check_edges(cs, qa, qb, policy=GPRM_EDGES_ALL_STEPS):
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


def _attach_lazy(cs, ends, verts, nb, label, Q, kk, rounds=4):
    """The attachment of `_answer_queries` with fewer checks and the same
    answer.  Each round looks, per query, at the first (start, goal)
    neighbour pair in nearest-first order whose vertices share a component
    and whose two attachment edges are not known to collide, and checks the
    unknown ones of those two edges; a query whose pair has both edges free
    is settled (every earlier pair lacks a shared component or has a
    colliding edge), a query without such a pair has no path.  After
    `rounds` rounds every unknown edge of the unsettled queries is checked.
    Returns (ok (2Q, kk) bool: edge checked and free, edges checked)."""
    import torch
    dev = verts.device
    lab = label[nb.clamp_min(0)].long()
    same = lab[:Q, :, None] == lab[Q:, None, :]                               # (Q, kk, kk)
    status = torch.where(nb >= 0, 0, 2).to(torch.int8)                        # 0 unknown, 1 free, 2 colliding
    rows = torch.arange(Q, device=dev)
    nchecked = 0
    for rnd in range(rounds + 1):
        col = status == 2
        cand = (same & ~col[:Q, :, None] & ~col[Q:, None, :]).reshape(Q, kk * kk)
        has = cand.any(1)
        first = torch.argmax(cand.to(torch.int8), dim=1)
        a, b = first // kk, first % kk
        ns = has & (status[rows, a] == 0)
        ng = has & (status[Q + rows, b] == 0)
        if rnd < rounds:
            er = torch.cat([rows[ns], Q + rows[ng]])
            ec = torch.cat([a[ns], b[ng]])
        else:
            open_ = ns | ng
            want = torch.cat([open_, open_])[:, None] & (status == 0)
            er, ec = torch.nonzero(want, as_tuple=True)
        if er.numel() == 0:
            break
        o = _longest_first(ends[er], verts[nb[er, ec].long()])
        er, ec = er[o], ec[o]
        ok = _check_edges(cs, ends[er], verts[nb[er, ec].long()]) == 0
        status[er, ec] = torch.where(ok, 1, 2).to(torch.int8)
        nchecked += int(er.numel())
    return status == 1, nchecked


def _longest_first(qa, qb):
    """Order of the edges qa[i] -> qb[i] by decreasing length: a batch whose
    long edges start first ends with short ones, so the check kernel's
    persistent warps finish together."""
    import torch
    return torch.argsort(torch.linalg.norm(qb - qa, dim=1), descending=True)


def _answer_queries(cs, graph, index, verts, i, j, good, label, starts, goals, k, ph=None, lazy=False):
    """Attaches every start and goal to its k nearest roadmap vertices by
    exactly checked edges, picks the first (start, goal) attachment pair in
    nearest-first order whose vertices share a component, and returns the
    forest paths through the roadmap, all on the device.  With lazy, only
    the attachment edges that decide this pair are checked
    (`_attach_lazy`, same pairs).  Returns (DevicePaths, attachment edges
    checked)."""
    import torch
    dev = verts.device
    Q = starts.shape[0]
    V = verts.shape[0]
    st = torch.as_tensor(starts, device=dev)
    gl = torch.as_tensor(goals, device=dev)
    if V == 0:
        z = torch.zeros(Q, dtype=torch.int32, device=dev)
        return DevicePaths(verts, z, z.long(), z[:0], starts, goals), 0
    ends = torch.cat([st, gl])
    kk = min(k, V)
    ph = ph or _Phases(False)
    nb = index.knn(kk, q=ends.T.contiguous())[0].long()                       # (2Q, kk)
    ph.mark("attach_knn")
    if lazy:
        ok, nconn = _attach_lazy(cs, ends, verts, nb, label, Q, kk)
    else:
        qa = ends[:, None, :].expand(-1, kk, -1).reshape(-1, ends.shape[1])
        ok = (_check_edges(cs, qa, verts[nb.reshape(-1)]) == 0).reshape(2 * Q, kk)
        nconn = 2 * Q * kk
    ph.mark("attach_edges")
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
    ph.mark("attach_match")
    parent, depth, levels = graph.forest(V, i, j, label, good)
    ph.mark("forest")
    length, off, flat_path = graph.paths(vs, vt, label, parent, depth)
    ph.mark("paths")
    if ph.on:
        ph.t["forest_levels"] = levels
    return DevicePaths(verts, length, off, flat_path, starts, goals), nconn


def verify_paths(cs, dp: DevicePaths):
    """Re-checks every edge of every path with the all-steps policy (each
    roadmap edge once, plus each path's start and goal segments); True if
    all are free."""
    import torch
    if len(dp) == 0:
        return True
    length, off, flat, verts = dp.length.long(), dp.off, dp.flat.long(), dp.verts
    dev = verts.device
    found = length > 0
    # roadmap segments: consecutive entries of the same path
    if flat.numel() > 1:
        owner = torch.repeat_interleave(torch.arange(len(dp), device=dev), length)
        same = owner[1:] == owner[:-1]
        u, v = flat[:-1][same], flat[1:][same]
        V = verts.shape[0]
        key = torch.unique(torch.minimum(u, v) * V + torch.maximum(u, v))
        ra, rb = verts[key // V], verts[key % V]
    else:
        ra = rb = verts[:0]
    st = torch.as_tensor(dp.starts, device=dev)[found]
    gl = torch.as_tensor(dp.goals, device=dev)[found]
    head = verts[flat[off[found]]]
    tail = verts[flat[off[found] + length[found] - 1]]
    qa = torch.cat([ra, st, tail])
    qb = torch.cat([rb, head, gl])
    o = _longest_first(qa, qb)
    return bool((_check_edges(cs, qa[o], qb[o], GPRM_EDGES_ALL_STEPS) == 0).all().item())



_WORKSPACES = {}


def _workspace(ndof: int):
    """The graph-operation and neighbour-index handles of a DOF, kept across
    planner calls so that their device buffers are allocated once."""
    ws = _WORKSPACES.get(ndof)
    if ws is None:
        ws = (RoadmapGraph(), NeighbourIndex(ndof))
        _WORKSPACES[ndof] = ws
    return ws


def _index_and_pairs(index, verts, k, radius=None, cap=64):
    """Indexes the roadmap vertices (the index is reused for the queries)
    and returns the undirected candidate edges (i < j, int64): the k
    nearest neighbours of every vertex, or with `radius` every pair closer
    than it (at most `cap` per vertex, in vertex order, like the
    reference's radius query get_near_vertices, prmsolver.cpp:2533-2574)."""
    import torch
    V = verts.shape[0]
    if V < 2:
        e = torch.empty(0, dtype=torch.int64, device=verts.device)
        if V:
            index.build(verts.T.contiguous())
        return e, e
    index.build(verts.T.contiguous())
    if radius is not None:
        _, idx, _ = index.radius(verts.T.contiguous(), float(radius), int(cap))
    else:
        idx, _ = index.knn(min(k, V - 1))
    rows = torch.arange(V, device=verts.device)[:, None].expand_as(idx)
    valid = (idx >= 0) & (idx != rows)
    a, b = rows[valid].long(), idx[valid].long()
    key = torch.unique(torch.minimum(a, b) * V + torch.maximum(a, b))
    return key // V, key % V


def _sample(scene, n, seed):
    """n configurations uniform in the joint box, drawn on the GPU (seeded)."""
    import torch
    g = torch.Generator(device="cuda:0")
    g.manual_seed(seed)
    lo = torch.tensor(scene.mins, device="cuda:0")
    hi = torch.tensor(scene.maxs, device="cuda:0")
    return lo + (hi - lo) * torch.rand((n, scene.ndof), device="cuda:0", generator=g)


def _cheapest_per_component(rest, la, lb, m):
    """The first m edges of `rest` (edge ids in weight order; la, lb the
    component labels of their ends, la != lb) at each component, counting
    both ends of every edge; each selected edge once."""
    import torch
    ends = torch.stack([la, lb], 1).reshape(-1)
    eid = rest.repeat_interleave(2)
    o = torch.argsort(ends, stable=True)                # by component, then weight
    ev = ends[o]
    rank = torch.arange(ev.numel(), device=ev.device) - torch.searchsorted(ev, ev)
    return torch.unique(eid[o][rank < m])


def _lazy_rounds(V, i64, j64, cost, check, components, max_rounds, first, growth, ph, length=None):
    """The rounds of `lazy_prm` over the candidate edges (i64[e], j64[e]):
    check(sel) gives the exact verdicts (True = free) of the edge ids sel,
    components(good) the component labels of the free-edge graph; with
    `length`, each round's batch is checked longest edge first; ph: the
    phase timer.  Returns (good uint8, checked bool, final labels, edges per
    round, free edges of round 1)."""
    import torch
    dev = i64.device
    E = int(i64.numel())
    good = torch.zeros(E, dtype=torch.uint8, device=dev)
    checked = torch.zeros(E, dtype=torch.bool, device=dev)
    # round 1: components are single vertices, so the selection is every
    # vertex's `first` cheapest candidate edges
    order = torch.argsort(cost, stable=True)
    label = torch.arange(V, dtype=torch.int32, device=dev)
    R = max(1, int(max_rounds))
    m, rounds, free1 = int(first), [], 0
    for rnd in range(R):
        rest = order[~checked[order]]
        la, lb = label[i64[rest]], label[j64[rest]]
        cross = la != lb
        rest, la, lb = rest[cross], la[cross], lb[cross]
        if rest.numel() == 0:
            break
        take = rest if rnd == R - 1 else _cheapest_per_component(rest, la, lb, m)
        if length is not None:
            take = take[torch.argsort(length[take], descending=True)]     # long edges first
        ph.mark("round1_select" if rnd == 0 else "round_select")
        ok = check(take)
        checked[take] = True
        good[take] = ok.to(torch.uint8)
        if rnd == 0:
            free1 = int(ok.sum().item())
        rounds.append(int(take.numel()))
        ph.mark("round1_edges" if rnd == 0 else "round_edges")
        label = components(good)
        ph.mark("components")
        m *= int(growth)
    return good, checked, label, rounds, free1


def plain_prm(cs, scene, starts, goals, n_samples, k=10, seed=0, profile=False, keep_roadmap=False,
              radius=None) -> PlanResult:
    """Eager GPU PRM: every vertex and every candidate edge checked (the k
    nearest neighbours, or with `radius` every pair within it).  With
    keep_roadmap, info["roadmap"] = (vertices, free-edge ends i, j) as host
    arrays (copied after the timed region), e.g. for results.store_plan."""
    import torch
    s0 = cs.stats()["edge_steps_nominal"]
    graph, index = _workspace(scene.ndof)
    ph = _Phases(profile)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ph.mark(None)
    q = _sample(scene, n_samples, seed)
    verts = q[_check_vertices(cs, q) == 0]
    ph.mark("vertices")
    i, j = _index_and_pairs(index, verts, k, radius)
    i, j = i.to(torch.int32), j.to(torch.int32)
    ph.mark("knn")
    good = (_check_edges(cs, verts[i.long()], verts[j.long()]) == 0).to(torch.uint8)
    ph.mark("edges")
    V = verts.shape[0]
    label = _components(graph, V, i, j, good)
    ph.mark("components")
    dp, nconn = _answer_queries(cs, graph, index, verts, i, j, good, label, starts, goals, k, ph)
    ph.mark("queries")
    ok = verify_paths(cs, dp)
    ph.mark("verify")
    found = dp.found()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    info = {"verified": ok, "free_vertices": V, "candidate_edges": int(i.numel()),
            **({"phases_ms": ph.t} if profile else {})}
    if keep_roadmap:
        g = good.bool()
        info["roadmap"] = (verts.cpu().numpy(), i[g].cpu().numpy(), j[g].cpu().numpy())
    return PlanResult(found, dp, dt, int(i.numel()) + nconn,
                      int(cs.stats()["edge_steps_nominal"] - s0), n_samples, info)


def lazy_prm(cs, scene, starts, goals, n_samples, k=10, seed=0, mlp=None, prune=0.9, beta=4.0,
             max_rounds=4, first=1, growth=2, lazy_attach=True, profile=False, radius=None) -> PlanResult:
    """Batched lazy-Boruvka PRM (exact connectivity), optionally MLP-guided;
    the roadmap and its bookkeeping stay on the device.  max_rounds >= 1
    counts round 1 (with max_rounds = 2 the second round checks every
    edge between components of round 1); lazy_attach: the query attachment
    of `_attach_lazy`."""
    import torch
    s0 = cs.stats()["edge_steps_nominal"]
    graph, index = _workspace(scene.ndof)
    ph = _Phases(profile)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ph.mark(None)
    q = _sample(scene, n_samples, seed)
    pruned = 0
    if mlp is not None:
        keep = mlp.predict(q.T.contiguous()) <= prune
        pruned = int((~keep).sum().item())
        q = q[keep]
        ph.mark("predict_samples")
    verts = q[_check_vertices(cs, q) == 0]
    vchecks = int(q.shape[0])
    ph.mark("vertices")
    i64, j64 = _index_and_pairs(index, verts, k, radius)
    ph.mark("knn")
    i, j = i64.to(torch.int32), j64.to(torch.int32)
    V, E = verts.shape[0], int(i.numel())
    dev = verts.device
    length = torch.linalg.norm(verts[i64] - verts[j64], dim=1)
    if mlp is not None and E:
        mid = 0.5 * (verts[i64] + verts[j64])
        pe = mlp.predict(mid.T.contiguous())
        cost = length * (1.0 + beta * pe)
        ph.mark("predict_edges")
    else:
        cost = length
    good, checked, label, rounds, free1 = _lazy_rounds(
        V, i64, j64, cost,
        lambda sel: _check_edges(cs, verts[i64[sel]], verts[j64[sel]]) == 0,
        lambda good_: _components(graph, V, i, j, good_),
        max_rounds, first, growth, ph, length)
    dp, nconn = _answer_queries(cs, graph, index, verts, i, j, good, label, starts, goals, k, ph,
                                lazy=lazy_attach)
    ph.mark("queries")
    ok = verify_paths(cs, dp)
    ph.mark("verify")
    found = dp.found()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return PlanResult(found, dp, dt, int(checked.sum().item()) + nconn,
                      int(cs.stats()["edge_steps_nominal"] - s0), vchecks,
                      {"verified": ok, "free_vertices": V, "candidate_edges": E, "round1_edges": rounds[0] if rounds else 0,
                       "round1_free": free1, "later_edges": int(sum(rounds[1:])), "rounds": len(rounds),
                       "pruned": pruned, **({"phases_ms": ph.t} if profile else {})})


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
    """The exact checker as the arbiter of the predictor on held-out uniform
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


def calibrate_prune(cs, scene, mlp, free_rate=0.002, n=1 << 16, seed=0, lo=0.9, hi=0.999, device="cuda:0"):
    """The prune threshold that removes at most `free_rate` of the free
    configurations: the (1 - free_rate) quantile of the predictor's p over
    exactly checked free held-out samples, kept within [lo, hi].  Pruning a
    free sample costs connectivity (the planner then needs more samples to
    reach the same success rate), so the threshold follows the predictor's
    own confidence on free space instead of a fixed value."""
    import torch
    q = torch.tensor(np.ascontiguousarray(scenes.uniform_configs(scene, n, seed + 777).T), device=device)
    codes = torch.zeros(n, dtype=torch.int32, device=device)
    cs.check_configs_device(q, codes)
    p = mlp.predict(q)[codes == 0]
    if p.numel() == 0:
        return hi
    t = float(torch.quantile(p.float(), 1.0 - free_rate).item())
    return min(max(t, lo), hi)


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
                     first=1, max_rounds=4, prune=None):
    """Plain (eager) PRM against the lazy PRM without guidance and the
    learned-guided lazy PRM, on the same seeded queries.  Each run is
    repeated (`repeats` timed runs after one untimed) and the median is
    reported.  The lazy PRM has the eager PRM's connectivity on the same
    samples, so its success rate is the same by construction.  The learned
    PRM prunes samples, which can change the roadmap: it runs on
    n_samples, then on 1.125x, 1.25x, ... samples until its success rate
    reaches the plain planner's, and the time of that run is the one
    compared ("equal success rate").  prune None: the threshold of
    `calibrate_prune` (at most 0.2 % of the free configurations pruned)."""
    starts, goals = make_queries(cs, scene, n_queries, seed + 17)
    out = {}
    plain = _median_run(lambda: plain_prm(cs, scene, starts, goals, n_samples, k, seed), repeats)
    out["plain"] = _summary(plain)
    lazy = _median_run(lambda: lazy_prm(cs, scene, starts, goals, n_samples, k, seed, first=first,
                                        max_rounds=max_rounds), repeats)
    out["lazy"] = _summary(lazy)
    if mlp is not None:
        if prune is None:
            prune = calibrate_prune(cs, scene, mlp, seed=seed)
        target = float(plain.success.mean())
        n, tries = n_samples, []
        for _ in range(8):
            r = _median_run(lambda: lazy_prm(cs, scene, starts, goals, n, k, seed, mlp=mlp, prune=prune,
                                             first=first, max_rounds=max_rounds), repeats)
            tries.append({"samples": n, "success_rate": float(r.success.mean()), "time_to_path_ms": 1e3 * r.time_to_path})
            if r.success.mean() >= target:
                break
            n = int(n * 1.125)
        out["learned"] = dict(_summary(r), samples=n, sample_search=tries,
                              success_matched=bool(r.success.mean() >= target))
        out["learned_over_plain_time"] = out["learned"]["time_to_path_ms"] / out["plain"]["time_to_path_ms"]
        out["learned_over_lazy_time"] = out["learned"]["time_to_path_ms"] / out["lazy"]["time_to_path_ms"]
        out["predictor_errors"] = predictor_errors(cs, scene, mlp, seed=seed, prune=prune)
        out["prune_threshold"] = prune
    out["lazy_over_plain_time"] = out["lazy"]["time_to_path_ms"] / out["plain"]["time_to_path_ms"]
    out["config"] = {"samples": n_samples, "queries": n_queries, "k": k, "seed": seed, "dq": float(cs.deltaq()),
                     "lazy_first": first, "lazy_rounds": max_rounds, "lazy_growth": 2, "lazy_attach": True}
    return out
