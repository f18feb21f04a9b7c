"""Seeded synthetic workloads with the shapes the benchmark configurations name.

``edge_workload`` builds the batched-edge workload of a PRM roadmap:
uniform samples in the joint box, the vertex check on the GPU, then the k
nearest free neighbours of every free sample (L2 in configuration space,
the metric the reference's planner connects by, prmsolver.cpp:2533-2574),
each undirected edge once.  The neighbour search runs on the GPU through
torch (chunked distance matrix + top-k); it prepares inputs and is not part
of any timed region.
"""
from __future__ import annotations

import numpy as np

from . import scenes
from .configspace import RobotConfigspace

HEADLINE = dict(kind="hull6", seed=0, n_samples=1 << 20, k=10, dq=0.01)


def knn_pairs(q, k: int, chunk: int = 2048):
    """Undirected k-nearest-neighbour pairs (i < j) of the rows of q, a
    (n, d) float32 CUDA tensor.  Returns two int64 CUDA tensors."""
    import torch
    n = q.shape[0]
    sq = (q * q).sum(1)
    out_i, out_j = [], []
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        d2 = sq[s:e, None] + sq[None, :] - 2.0 * (q[s:e] @ q.T)
        d2[torch.arange(e - s, device=q.device), torch.arange(s, e, device=q.device)] = float("inf")
        kk = min(k, n - 1)
        idx = torch.topk(d2, kk, dim=1, largest=False).indices
        rows = torch.arange(s, e, device=q.device)[:, None].expand(-1, kk)
        out_i.append(rows.reshape(-1))
        out_j.append(idx.reshape(-1))
    i = torch.cat(out_i)
    j = torch.cat(out_j)
    a = torch.minimum(i, j)
    b = torch.maximum(i, j)
    key = torch.unique(a * n + b)
    return key // n, key % n


def edge_workload(kind: str = "hull6", seed: int = 0, n_samples: int = 1 << 20, k: int = 10,
                  dq: float = 0.01, device: str = "cuda:0", scene=None):
    """Returns dict(scene, space, qs, qe (ndof, E) float32 CUDA SoA, n_free)."""
    import torch
    sc = scene if scene is not None else scenes.make_scene(kind, seed)
    cs = RobotConfigspace(sc, dq=dq)
    cs.init()
    q_np = scenes.uniform_configs(sc, n_samples, seed + 1000)
    q_soa = torch.tensor(np.ascontiguousarray(q_np.T), device=device)
    codes = torch.zeros(n_samples, dtype=torch.int32, device=device)
    cs.check_configs_device(q_soa, codes)
    torch.cuda.synchronize()
    free = torch.nonzero(codes == 0).squeeze(1)
    qf = q_soa[:, free].T.contiguous()
    i, j = knn_pairs(qf, k)
    qs = qf[i].T.contiguous()
    qe = qf[j].T.contiguous()
    return dict(scene=sc, space=cs, qs=qs, qe=qe, n_free=int(free.numel()), n_samples=n_samples,
                q_soa=q_soa, codes=codes)
