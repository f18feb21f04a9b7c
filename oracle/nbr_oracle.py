"""CPU restatement of the neighbour search (test infrastructure only).

TEST INFRASTRUCTURE ONLY: the checker of gprm_nbr_radius / gprm_nbr_knn.

Distance as in get_near_vertices (prm/src/lib/prm/prmsolver.cpp:2533-2574):
float32 d = x_j - q_j, s = s + d*d over the joints in order (numpy float32
arithmetic rounds after every operation, like the kernels compiled without
FMA contraction); a node is within D when s < D*D (D*D rounded to float,
prmsolver.cpp:71); dist = sqrt(s) in float32.
"""
from __future__ import annotations

import numpy as np


def dist2(x: np.ndarray, q: np.ndarray) -> np.ndarray:
    """x: (n, ndof) float32 nodes, q: (ndof,) -> (n,) float32 squared distances."""
    s = np.zeros(x.shape[0], np.float32)
    for j in range(x.shape[1]):
        d = (x[:, j] - np.float32(q[j])).astype(np.float32)
        s = (s + (d * d).astype(np.float32)).astype(np.float32)
    return s


def radius(x: np.ndarray, q: np.ndarray, D: float, cap: int):
    """Per query: ascending node indices within D (first `cap`) and distances."""
    D2 = np.float32(np.float32(D) * np.float32(D))
    out = []
    for t in range(q.shape[0]):
        s = dist2(x, q[t])
        hit = np.nonzero(s < D2)[0][:cap]
        out.append((hit.astype(np.int32), np.sqrt(s[hit]).astype(np.float32)))
    return out


def knn(x: np.ndarray, q: np.ndarray, k: int, exclude=None):
    """k nearest by (s, index); NaN distances sort last; exclude[t] is a
    node index to skip for query t (or None)."""
    idx = np.full((q.shape[0], k), -1, np.int32)
    dist = np.full((q.shape[0], k), np.inf, np.float32)
    for t in range(q.shape[0]):
        s = dist2(x, q[t]).copy()
        s[np.isnan(s)] = np.inf
        ids = np.arange(x.shape[0])
        if exclude is not None:
            keep = ids != exclude[t]
            s, ids = s[keep], ids[keep]
        order = np.lexsort((ids, s))[:k]
        idx[t, :len(order)] = ids[order]
        dist[t, :len(order)] = np.sqrt(s[order])
    return idx, dist
