"""Batched sampling near roadmap nodes (gprm_sample_near of the C ABI).

The reference draws one candidate at a time near a stored node, accepting it
with probability 1/(1+surrnum)^p and checking it with a host indicator(q)
call (get_random_nodes, prm/src/lib/prm/prmsolver.cpp:2585-2698).  Here a
batch of candidates is drawn in one kernel (Philox counter-based random
numbers, so (seed, t) fixes candidate t) and the accepted ones are checked
in one batched vertex check; the result is the first `num` accepted, free
candidates in t order, independent of the batch size.  Given the
reference's block storage (`blocks` = (pos, num) int32 CUDA tensors of its
non-empty blocks, prmsolver.h:29-59) the parent is drawn as there, a block
first and then a node in it (gprm_sample_near_blocks); without, uniformly
among the nodes.
"""
from __future__ import annotations

import ctypes as C

from . import _abi
from .configspace import GprmError, _current_stream


def candidates(nodes, surrnum, D: float, seed: int, t0: int, B: int, power: int = 3, stream=None, blocks=None):
    """nodes (ndof, n) float32 and surrnum (n,) int32 CUDA tensors ->
    (q (ndof, B), parent (B,) int32; -1 = dismissed)."""
    import torch
    lib = _abi.load_library()
    ndof, n = int(nodes.shape[0]), int(nodes.shape[1])
    q = torch.empty((ndof, B), dtype=torch.float32, device=nodes.device)
    par = torch.empty(B, dtype=torch.int32, device=nodes.device)
    st = stream if stream is not None else _current_stream()
    if blocks is None:
        rc = lib.gprm_sample_near(ndof, C.c_void_p(nodes.data_ptr()), n, n, C.c_void_p(surrnum.data_ptr()),
                                  int(power), float(D), int(seed), int(t0), int(B), C.c_void_p(q.data_ptr()), B,
                                  C.c_void_p(par.data_ptr()), C.c_void_p(st))
    else:
        pos, num = blocks
        rc = lib.gprm_sample_near_blocks(ndof, C.c_void_p(nodes.data_ptr()), n, n, C.c_void_p(pos.data_ptr()),
                                         C.c_void_p(num.data_ptr()), int(pos.numel()),
                                         C.c_void_p(surrnum.data_ptr()), int(power), float(D), int(seed), int(t0),
                                         int(B), C.c_void_p(q.data_ptr()), B, C.c_void_p(par.data_ptr()),
                                         C.c_void_p(st))
    if rc != 0:
        raise GprmError(rc, "gprm_sample_near failed")
    return q, par


def sample_near(cs, nodes, surrnum, num: int, D: float, seed: int, power: int = 3, batch: int = 1 << 16,
                max_batches: int = 1000, blocks=None):
    """The first `num` accepted, collision-free candidates in t order:
    (q (ndof, num) CUDA tensor, parents (num,), candidates consumed)."""
    import torch
    outs_q, outs_p, got, t0 = [], [], 0, 0
    for _ in range(max_batches):
        q, par = candidates(nodes, surrnum, D, seed, t0, batch, power, blocks=blocks)
        acc = torch.nonzero(par >= 0).squeeze(1)
        free = torch.zeros(batch, dtype=torch.bool, device=q.device)
        if acc.numel():
            codes = torch.empty(acc.numel(), dtype=torch.int32, device=q.device)
            cs.check_configs_device(q[:, acc].contiguous(), codes)
            free[acc] = codes == 0
        sel = torch.nonzero(free).squeeze(1)[:num - got]
        outs_q.append(q[:, sel])
        outs_p.append(par[sel])
        got += int(sel.numel())
        if got >= num:
            return torch.cat(outs_q, 1), torch.cat(outs_p), t0 + int(sel[-1].item()) + 1
        t0 += batch
    return torch.cat(outs_q, 1), torch.cat(outs_p), t0
