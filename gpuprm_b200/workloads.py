"""Seeded synthetic workloads with the shapes the benchmark configurations name.

``edge_workload`` builds the batched-edge workload of a PRM roadmap:
uniform samples in the joint box, the vertex check on the GPU, then the k
nearest free neighbours of every free sample (L2 in configuration space,
the metric the reference's planner connects by, prmsolver.cpp:2533-2574),
each undirected edge once.  The neighbour search runs on the GPU in the
library's own kNN kernel (gprm_nbr_knn); it prepares inputs and is not part
of any timed region.
"""
from __future__ import annotations

import numpy as np

from . import scenes
from .configspace import RobotConfigspace

HEADLINE = dict(kind="hull6", seed=0, n_samples=1 << 20, k=10, dq=0.01)


def knn_pairs(q, k: int):
    """Undirected k-nearest-neighbour pairs (i < j) of the rows of q, a
    (n, d) float32 CUDA tensor, by the library's exact grid kNN kernel
    (gprm_nbr_knn).  Returns two int64 CUDA tensors."""
    from .neighbours import knn_pairs as _knn
    return _knn(q.T.contiguous(), k)


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


MANY = dict(problems=256, dof=(4, 7), obstacles=(8, 128), samples_log2=(14, 18), radius=(0.4, 0.8),
            edge_sources=None, k=10, dq=0.01)


def batch_workload(seed: int = 0, problems: int = MANY["problems"], samples_log2=MANY["samples_log2"],
                   radius=MANY["radius"], edge_sources=MANY["edge_sources"], k: int = MANY["k"],
                   dq: float = MANY["dq"], device: str = "cuda:0"):
    """Many independent problems (``scenes.make_mixed``: DOF 4-7, 8-128
    obstacles), each with 2^U[lo,hi] uniform samples and a connection
    radius U[0.4, 0.8].  Edges: the k nearest free neighbours of every free
    sample of each problem (of its first ``edge_sources`` free samples when
    given), each undirected edge once, every edge longer than the radius
    cut back to the radius along its direction (the planner connects within
    the radius).  Everything is built and packed on the device.  Returns
    dict(spaces, scenes, q, qs, qe (7, total) float32 CUDA SoA with rows
    ndof..6 zero, offs_v, offs_e (numpy), n_free)."""
    import torch
    from .batch import MAX_DOF, offsets_of
    rng = np.random.default_rng(seed)
    spaces, scs, qv, qa, qb, n_free = [], [], [], [], [], []
    for p in range(problems):
        sc = scenes.make_mixed(seed * 100003 + p)
        cs = RobotConfigspace(sc, dq=dq)
        cs.init()
        n = int(round(2.0 ** rng.uniform(*samples_log2)))
        r = float(rng.uniform(*radius))
        q = scenes.uniform_configs(sc, n, seed * 7 + p)
        qd = torch.tensor(np.ascontiguousarray(q.T), device=device)
        codes = torch.zeros(n, dtype=torch.int32, device=device)
        cs.check_configs_device(qd, codes)
        free = torch.nonzero(codes == 0).squeeze(1)
        if edge_sources is not None:
            free = free[:edge_sources]
        qf = qd[:, free].T.contiguous()
        if qf.shape[0] >= 2:
            i, j = knn_pairs(qf, k)
            a, b = qf[i], qf[j]
            d = b - a
            L = torch.linalg.vector_norm(d, dim=1, keepdim=True)
            scale = torch.clamp(r / torch.clamp(L, min=1e-30), max=1.0)
            b = a + d * scale
        else:
            a = b = qf[:0]
        spaces.append(cs)
        scs.append(sc)
        qv.append(qd)
        qa.append(a.T)
        qb.append(b.T)
        n_free.append(int((codes == 0).sum().item()))
    offs_v = offsets_of([x.shape[1] for x in qv])
    offs_e = offsets_of([x.shape[1] for x in qa])

    def pack(parts, offs):
        out = torch.zeros((MAX_DOF, int(offs[-1])), dtype=torch.float32, device=device)
        for x, o in zip(parts, offs[:-1]):
            out[:x.shape[0], int(o):int(o) + x.shape[1]] = x
        return out
    return dict(spaces=spaces, scenes=scs, q=pack(qv, offs_v), qs=pack(qa, offs_e), qe=pack(qb, offs_e),
                offs_v=offs_v, offs_e=offs_e, n_free=n_free)
