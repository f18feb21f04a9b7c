"""Neighbour search: the CPU restatement pinned against the reference
planner's own get_near_vertices (prmsolver.cpp:2533-2574, compiled from its
sources into oracle/_ref/libnbr_ref.so), and the device kernels checked
against the restatement bit for bit (indices, float32 distances)."""
import ctypes as C
import os

import numpy as np
import pytest

import nbr_oracle as NO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnbr_ref.so")


def _points(n, ndof, seed, lo=-np.pi, hi=np.pi):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (n, ndof)).astype(np.float32)


def test_oracle_radius_small_cases():
    x = np.array([[0, 0], [1, 0], [0, 1], [0.5, 0.5]], np.float32)
    q = np.array([[0, 0]], np.float32)
    (hit, d), = NO.radius(x, q, 1.0, 10)
    assert hit.tolist() == [0, 3]          # (1,0) and (0,1) are at exactly D: s < D*D excludes them
    assert d[0] == 0.0 and abs(d[1] - np.float32(np.sqrt(0.5))) == 0
    (hit, _), = NO.radius(x, q, 1.0001, 2)
    assert hit.tolist() == [0, 1]          # the first cap in index order


def test_oracle_knn_ties_and_exclusion():
    x = np.array([[0.0], [1.0], [-1.0], [2.0], [np.nan]], np.float32)
    idx, dist = NO.knn(x, x[:1], 3, exclude=[0])
    assert idx.tolist() == [[1, 2, 3]]     # tie at distance 1 broken by index
    idx, _ = NO.knn(x, x[:1], 5, exclude=[0])
    assert idx.tolist() == [[1, 2, 3, 4, -1]]   # NaN distance sorts last


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref/libnbr_ref.so not built")
@pytest.mark.parametrize("ndof,D,H", [(4, 0.9, 1.0), (6, 1.4, 0.5)])
def test_oracle_matches_reference_get_near_vertices(ndof, D, H):
    lib = C.CDLL(REF_LIB)
    x = _points(3000, ndof, 1)
    q = _points(40, ndof, 2)
    nbuf = 3000
    counts = np.zeros(len(q), np.int32)
    idx = np.zeros((len(q), nbuf), np.int32)
    dist = np.zeros((len(q), nbuf), np.float32)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = lib.ref_near_vertices(ndof, P(x), len(x), P(q), len(q), C.c_float(D), C.c_float(H), nbuf, P(counts),
                               P(idx), P(dist))
    assert rc == 0
    want = NO.radius(x, q, D, nbuf)
    assert counts.sum() > 0
    for t in range(len(q)):
        got_i = idx[t, :counts[t]]
        order = np.argsort(got_i)
        np.testing.assert_array_equal(got_i[order], want[t][0])
        np.testing.assert_array_equal(dist[t, :counts[t]][order], want[t][1])


@pytest.mark.gpu
@pytest.mark.parametrize("ndof,n,m,D,cap", [(4, 5000, 300, 1.0, 64), (6, 20000, 200, 1.6, 4096), (7, 100, 50, 10.0, 7)])
def test_gpu_radius_matches_oracle(ndof, n, m, D, cap):
    import torch
    from gpuprm_b200.neighbours import NeighbourIndex
    x = _points(n, ndof, 3)
    q = _points(m, ndof, 4)
    ix = NeighbourIndex(ndof)
    xd = torch.tensor(np.ascontiguousarray(x.T), device="cuda:0")
    ix.build(xd)
    counts, idx, dist = ix.radius(torch.tensor(np.ascontiguousarray(q.T), device="cuda:0"), D, cap)
    torch.cuda.synchronize()
    counts, idx, dist = counts.cpu().numpy(), idx.cpu().numpy(), dist.cpu().numpy()
    want = NO.radius(x, q, D, cap)
    for t in range(m):
        np.testing.assert_array_equal(idx[t, :counts[t]], want[t][0])
        np.testing.assert_array_equal(dist[t, :counts[t]], want[t][1])


@pytest.mark.gpu
@pytest.mark.parametrize("ndof,n,k,spread", [(4, 8000, 10, "uniform"), (6, 30000, 16, "uniform"),
                                             (3, 5000, 32, "clustered"), (2, 40, 32, "uniform"),
                                             (7, 3000, 8, "duplicates")])
def test_gpu_knn_self_matches_oracle(ndof, n, k, spread):
    import torch
    from gpuprm_b200.neighbours import NeighbourIndex
    rng = np.random.default_rng(5)
    if spread == "uniform":
        x = _points(n, ndof, 6)
    elif spread == "clustered":
        c = rng.uniform(-3, 3, (8, ndof))
        x = (c[rng.integers(0, 8, n)] + rng.normal(0, 0.05, (n, ndof))).astype(np.float32)
    else:   # many exact duplicates: ties resolved by index
        x = np.round(_points(n, ndof, 7), 1).astype(np.float32)
        x[::3] = x[0]
    ix = NeighbourIndex(ndof)
    ix.build(torch.tensor(np.ascontiguousarray(x.T), device="cuda:0"))
    idx, dist = ix.knn(k)
    torch.cuda.synchronize()
    sample = rng.choice(n, min(n, 400), replace=False)
    want_i, want_d = NO.knn(x, x[sample], k, exclude=sample)
    np.testing.assert_array_equal(idx.cpu().numpy()[sample], want_i)
    np.testing.assert_array_equal(dist.cpu().numpy()[sample], want_d)


@pytest.mark.gpu
def test_gpu_knn_external_queries_and_redo_path():
    """Queries outside the nodes' extent cannot be settled by the grid and
    go through the full scan; both paths give the oracle's answer."""
    import torch
    from gpuprm_b200.neighbours import NeighbourIndex
    x = _points(6000, 5, 8)
    q = np.concatenate([_points(200, 5, 9), _points(50, 5, 10, 5.0, 9.0)]).astype(np.float32)
    ix = NeighbourIndex(5)
    ix.build(torch.tensor(np.ascontiguousarray(x.T), device="cuda:0"))
    idx, dist = ix.knn(12, q=torch.tensor(np.ascontiguousarray(q.T), device="cuda:0"))
    torch.cuda.synchronize()
    assert ix.redo_count() >= 50
    want_i, want_d = NO.knn(x, q, 12)
    np.testing.assert_array_equal(idx.cpu().numpy(), want_i)
    np.testing.assert_array_equal(dist.cpu().numpy(), want_d)
