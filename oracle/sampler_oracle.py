"""CPU restatement of the batched near-node sampler (test infrastructure).

TEST INFRASTRUCTURE ONLY: the checker of gprm_sample_near.

Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011) written out from the
paper in numpy (pinned by the published known-answer vectors in
tests/test_sampler.py), and candidate generation as get_random_nodes
(prm/src/lib/prm/prmsolver.cpp:2585-2624): parent m uniform, accepted when
r <= (2^31-1) // (1+surrnum[m])^power, q = (node - D) + (2*D) * (r'/2^31) in
float32 arithmetic.  With the reference's block storage (block_pos,
block_num; prmsolver.cpp:2589-2597) the parent is drawn in two steps as
there: block b = r0 % nblocks, then slot block_pos[b] + r9 % block_num[b].
"""
from __future__ import annotations

import numpy as np

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised over arrays of counters; returns four uint32 arrays."""
    c = [np.asarray(x, np.uint64) & _MASK for x in (c0, c1, c2, c3)]
    k0 = np.uint64(k0) & _MASK
    k1 = np.uint64(k1) & _MASK
    for _ in range(10):
        p0 = np.uint64(M0) * c[0]
        p1 = np.uint64(M1) * c[2]
        c = [((p1 >> np.uint64(32)) ^ c[1] ^ k0) & _MASK, p1 & _MASK,
             ((p0 >> np.uint64(32)) ^ c[3] ^ k1) & _MASK, p0 & _MASK]
        k0 = (k0 + np.uint64(W0)) & _MASK
        k1 = (k1 + np.uint64(W1)) & _MASK
    return [x.astype(np.uint32) for x in c]


def candidates(nodes, surrnum, power, D, seed, t0, B, block_pos=None, block_num=None):
    """nodes (n, ndof) float32 -> (q (B, ndof) float32, parent (B,) int, -1 dismissed).
    With block_pos/block_num the nodes are storage slots and the parent is
    drawn block first (empty blocks and slots outside the nodes dismiss,
    q = 0 there)."""
    nodes = np.asarray(nodes, np.float32)
    n, ndof = nodes.shape
    t = np.arange(t0, t0 + B, dtype=np.uint64)
    tl, th = t & _MASK, t >> np.uint64(32)
    k0, k1 = seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF
    z = np.zeros(B, np.uint64)
    blocks = [philox4x32_10(tl, th, z + np.uint64(j), z, k0, k1) for j in range(3)]
    r = [x >> np.uint32(1) for blk in blocks for x in blk][:10]
    bad = np.zeros(B, bool)
    if block_pos is not None:
        bp, bn = np.asarray(block_pos, np.int64), np.asarray(block_num, np.int64)
        b = (r[0] % np.uint32(len(bp))).astype(np.int64)
        cnt = bn[b]
        bad = cnt <= 0
        m = bp[b] + (r[9].astype(np.int64) % np.maximum(cnt, 1))
        bad |= (m < 0) | (m >= n)
        m = np.where(bad, 0, m)
    else:
        m = (r[0] % np.uint32(n)).astype(np.int64)
    x = 1 + np.maximum(np.asarray(surrnum, np.int64)[m], 0)
    xp = np.ones(B, np.int64)
    for _ in range(power):
        xp = np.where(xp > (1 << 40), xp, xp * x)
    accept = r[1].astype(np.int64) <= (2147483647 // xp)
    q = np.empty((B, ndof), np.float32)
    twoD = np.float32(2.0) * np.float32(D)
    for j in range(ndof):
        u = (r[2 + j].astype(np.float32) / np.float32(2147483648.0)).astype(np.float32)
        q[:, j] = ((nodes[m, j] - np.float32(D)).astype(np.float32) + (twoD * u).astype(np.float32)).astype(np.float32)
    q[bad] = 0.0
    return q, np.where(accept & ~bad, m, -1)


def sample_near(nodes, surrnum, power, D, seed, num, is_free, batch=4096, max_batches=1000, block_pos=None,
                block_num=None):
    """The first `num` accepted candidates, in t order, that is_free(q (k, ndof))
    reports free: (q (num, ndof), parents, candidates consumed)."""
    out_q, out_p, t0 = [], [], 0
    got = 0
    for _ in range(max_batches):
        q, par = candidates(nodes, surrnum, power, D, seed, t0, batch, block_pos, block_num)
        acc = np.nonzero(par >= 0)[0]
        free = np.zeros(batch, bool)
        if len(acc):
            free[acc] = is_free(q[acc])
        sel = np.nonzero(free)[0][:num - got]
        out_q.append(q[sel])
        out_p.append(par[sel])
        got += len(sel)
        if got >= num:
            return np.concatenate(out_q), np.concatenate(out_p), t0 + (sel[-1] + 1 if len(sel) else batch)
        t0 += batch
    return np.concatenate(out_q), np.concatenate(out_p), t0
