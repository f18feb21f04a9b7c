"""CPU restatement of the roadmap graph operations (test infrastructure).

TEST INFRASTRUCTURE ONLY: the checker of the gprm_graph_* kernels.

* components: label = smallest vertex of the component;
* forest: level-synchronous breadth-first forest from each component's
  label vertex; the parent of a vertex is its smallest neighbour on the
  previous level;
* dijkstra: Dijkstra as in do_dijkstra (prm/src/lib/prm/prmsolver.cpp:
  2805-2846) with float32 path sums accumulated from the source; parent =
  smallest neighbour u with dist[u] + w == dist[v].
"""
from __future__ import annotations

import heapq

import numpy as np


def components(V: int, eu, ev) -> np.ndarray:
    parent = list(range(V))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in zip(eu, ev):
        ra, rb = find(int(a)), find(int(b))
        if ra != rb:
            if ra < rb:
                ra, rb = rb, ra
            parent[ra] = rb
    return np.array([find(i) for i in range(V)], np.int32)


def forest(V: int, eu, ev, label):
    adj = [[] for _ in range(V)]
    for a, b in zip(eu, ev):
        adj[int(a)].append(int(b))
        adj[int(b)].append(int(a))
    INF = np.iinfo(np.int32).max
    depth = np.full(V, INF, np.int64)
    parent = np.full(V, -1, np.int64)
    frontier = [i for i in range(V) if label[i] == i]
    for i in frontier:
        depth[i] = 0
    level = 0
    while frontier:
        cand = {}
        for u in frontier:
            for v in adj[u]:
                if depth[v] == INF:
                    cand[v] = min(cand.get(v, INF), u)
        for v, u in cand.items():
            depth[v] = level + 1
            parent[v] = u
        frontier = sorted(cand)
        level += 1
    return parent, depth


def forest_path(parent, depth, s, t):
    a, b = [s], [t]
    while depth[a[-1]] > depth[b[-1]]:
        a.append(int(parent[a[-1]]))
    while depth[b[-1]] > depth[a[-1]]:
        b.append(int(parent[b[-1]]))
    while a[-1] != b[-1]:
        a.append(int(parent[a[-1]]))
        b.append(int(parent[b[-1]]))
    return a + b[-2::-1]


def dijkstra(V: int, eu, ev, w, src):
    adj = [[] for _ in range(V)]
    for a, b, x in zip(eu, ev, w):
        adj[int(a)].append((int(b), np.float32(x)))
        adj[int(b)].append((int(a), np.float32(x)))
    dist = np.full(V, np.inf, np.float32)
    dist[src] = np.float32(0)
    heap = [(np.float32(0), src)]
    done = np.zeros(V, bool)
    while heap:
        d, u = heapq.heappop(heap)
        if done[u] or d > dist[u]:
            continue
        done[u] = True
        for v, x in adj[u]:
            nd = np.float32(dist[u] + x)
            if nd < dist[v]:
                dist[v] = nd
                heapq.heappush(heap, (nd, v))
    parent = np.full(V, -1, np.int64)
    parent[src] = src
    for v in range(V):
        if v == src or not np.isfinite(dist[v]):
            continue
        best = None
        for u, x in adj[v]:
            if np.isfinite(dist[u]) and np.float32(dist[u] + x) == dist[v]:
                best = u if best is None else min(best, u)
        parent[v] = best if best is not None else -1
    return dist, parent
