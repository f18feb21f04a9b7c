"""The near-node sampler pinned distributionally to the reference's own
get_random_nodes (prm/src/lib/prm/prmsolver.cpp:2585-2624), compiled from
its sources into oracle/_ref/libnbr_ref.so (ref_random_nodes).

Both draw from the same roadmap: nodes on a lattice (spacing 1, so the
boxes of half-width D = 0.2 around them are disjoint and every sample names
its parent) stored by the reference's insert() in blocks keyed by joint 0,
with slabs of very different sizes (so the block-first parent draw weighs
nodes unequally) and surrnum 0..3 (acceptance 1/(1+s)^3), and a wall at
q0 = 3.55 that the space reports as collision (cutting one slab's boxes).
Over about 10^6 proposals on each side:
  * the parents follow the reference's weights (chi-square against the
    exact probabilities, and a two-sample contingency test reference vs
    oracle restatement);
  * the offsets q - parent are uniform in [-D, D] away from the wall (KS),
    and the two sides' offsets agree (two-sample KS), at the wall too;
  * the fraction of proposals dismissed by the surrnum test matches.
The GPU kernel equals the restatement bit for bit (tests/test_sampler.py),
so this pins it too.  The uniform-parent draw of gprm_sample_near is shown
to differ from the reference on such a roadmap: the block-storage entry
point is the drop-in.
"""
import ctypes as C
import os

import numpy as np
import pytest

import sampler_oracle as SO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnbr_ref.so")
pytestmark = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref/libnbr_ref.so not built")

NDOF, D, H, WALL, POWER = 4, 0.2, 1.0, 3.55, 3
SLABS = (3, 10, 40, 100, 300, 600)     # nodes per joint-0 slab; 300 and 600 fill several 256-node blocks
NUM = 300_000                            # free samples drawn on each side (~10^6 proposals)


def _roadmap():
    rng = np.random.default_rng(11)
    lat = np.stack(np.meshgrid(*[np.arange(9)] * 3, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    xs = []
    for s, cnt in enumerate(SLABS):
        pick = rng.permutation(len(lat))[:cnt]
        xs.append(np.concatenate([np.full((cnt, 1), s + 0.5, np.float32), lat[pick]], 1))
    x = np.concatenate(xs)[rng.permutation(sum(SLABS))]
    surr = rng.integers(0, 4, len(x)).astype(np.int32)
    return np.ascontiguousarray(x), surr


def _reference(x, surr, seed):
    lib = C.CDLL(REF_LIB)
    lib.ref_random_nodes.restype = C.c_int
    n = len(x)
    q = np.zeros((NUM, NDOF), np.float32)
    slot = np.zeros(n, np.int32)
    bpos = np.zeros(2 * n + 64, np.int32)
    bnum = np.zeros(2 * n + 64, np.int32)
    nb = C.c_int(0)
    cnt = np.zeros(4, np.int64)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = lib.ref_random_nodes(NDOF, P(x), n, P(surr), C.c_float(H), C.c_float(D), C.c_float(WALL), seed, NUM,
                              P(q), P(slot), P(bpos), P(bnum), C.byref(nb), P(cnt))
    assert rc == 0
    return q, slot, bpos[:nb.value], bnum[:nb.value], cnt


def _parents(q, x):
    """The node whose box holds each sample (boxes are disjoint)."""
    from scipy.spatial import cKDTree
    d, i = cKDTree(x.astype(np.float64)).query(q.astype(np.float64), p=np.inf)
    assert (d <= D * (1 + 1e-5)).all()
    return i


def _expected(x, surr, bpos, bnum, slot):
    """The reference's probability of each node as the parent of a free
    sample: block weight x surrnum acceptance x the free part of its box."""
    nonempty = bnum > 0
    w_block = np.zeros(len(x))
    for p, c in zip(bpos[nonempty], bnum[nonempty]):
        inside = (slot >= p) & (slot < p + c)
        w_block[inside] = 1.0 / (nonempty.sum() * c)
    acc = np.array([(2147483647 // (1 + int(s)) ** POWER + 1) / 2147483648.0 for s in surr])
    lo = x[:, 0] - D
    free = np.clip((WALL - lo) / (2 * D), 0.0, 1.0)
    p = w_block * acc * free
    return p / p.sum(), float((w_block * (1 - acc)).sum()), float((w_block * acc * (1 - free)).sum())


@pytest.fixture(scope="module")
def draws():
    x, surr = _roadmap()
    rq, slot, bpos, bnum, cnt = _reference(x, surr, seed=7)
    n_slots = int((bpos + 256).max())
    storage = np.zeros((n_slots, NDOF), np.float32)
    storage[slot] = x
    ssurr = np.zeros(n_slots, np.int32)
    ssurr[slot] = surr
    keep = bnum > 0
    free = lambda qq: qq[:, 0] <= np.float32(WALL)
    oq, opar, used = SO.sample_near(storage, ssurr, POWER, D, 12345, NUM, free, batch=1 << 16,
                                    block_pos=bpos[keep], block_num=bnum[keep])
    # proposals the surrnum test dismissed, on the oracle's side
    _, par_all = SO.candidates(storage, ssurr, POWER, D, 12345, 0, int(used), bpos[keep], bnum[keep])
    return dict(x=x, surr=surr, slot=slot, bpos=bpos, bnum=bnum, cnt=cnt, rq=rq, oq=oq, opar=opar, used=int(used),
                o_dismissed=int((par_all < 0).sum()), storage=storage, ssurr=ssurr)


def test_reference_roadmap_has_unequal_blocks(draws):
    bnum = draws["bnum"]
    sizes = sorted(int(c) for c in bnum if c > 0)
    assert sizes[0] <= 3 and sizes[-1] == 256 and len(sizes) >= 9
    assert draws["cnt"][0] >= 900_000                   # about 10^6 reference proposals


def test_parents_follow_the_reference_weights(draws):
    from scipy.stats import chi2_contingency, chisquare
    x = draws["x"]
    p, _, _ = _expected(x, draws["surr"], draws["bpos"], draws["bnum"], draws["slot"])
    ref = np.bincount(_parents(draws["rq"], x), minlength=len(x))
    slot_to_node = np.full(len(draws["storage"]), -1)
    slot_to_node[draws["slot"]] = np.arange(len(x))
    ours = np.bincount(slot_to_node[draws["opar"]], minlength=len(x))
    assert (slot_to_node[draws["opar"]] >= 0).all()
    np.testing.assert_array_equal(_parents(draws["oq"], x), slot_to_node[draws["opar"]])
    # pool the rarely drawn nodes so every cell expects >= 20 samples
    order = np.argsort(p)
    groups = np.zeros(len(x), int)
    acc, g = 0.0, 0
    for i in order:
        groups[i] = g
        acc += p[i] * NUM
        if acc >= 20:
            g, acc = g + 1, 0.0
    G = groups.max() + 1
    pe = np.bincount(groups, p, G)
    for obs in (ref, ours):
        o = np.bincount(groups, obs, G)
        assert o.sum() == NUM
        assert chisquare(o, pe * NUM).pvalue > 1e-4
    table = np.stack([np.bincount(groups, ref, G), np.bincount(groups, ours, G)])
    assert chi2_contingency(table).pvalue > 1e-4
    # the uniform-parent draw does not follow them
    uni = np.bincount(groups, (p > 0) * _expected_uniform(draws), G)
    assert chisquare(uni / uni.sum() * NUM, pe * NUM).pvalue < 1e-12


def _expected_uniform(draws):
    x, surr = draws["x"], draws["surr"]
    acc = np.array([(2147483647 // (1 + int(s)) ** POWER + 1) / 2147483648.0 for s in surr])
    free = np.clip((WALL - (x[:, 0] - D)) / (2 * D), 0.0, 1.0)
    return acc * free / (acc * free).sum()


def test_offsets_are_uniform_and_agree(draws):
    from scipy.stats import ks_2samp, kstest
    x = draws["x"]
    ro = (draws["rq"] - x[_parents(draws["rq"], x)]) / D
    oo = (draws["oq"] - x[_parents(draws["oq"], x)]) / D
    for j in range(NDOF):
        assert ks_2samp(ro[:, j], oo[:, j]).pvalue > 1e-4
    away = x[_parents(draws["rq"], x)][:, 0] != np.float32(3.5)
    oaway = x[_parents(draws["oq"], x)][:, 0] != np.float32(3.5)
    for j in range(NDOF):
        assert kstest(ro[away, j], "uniform", args=(-1, 2)).pvalue > 1e-4
        assert kstest(oo[oaway, j], "uniform", args=(-1, 2)).pvalue > 1e-4
    # in the slab cut by the wall joint 0 is uniform on the free part only
    assert ro[~away, 0].max() <= (WALL - 3.5) / D + 1e-5 and oo[~oaway, 0].max() <= (WALL - 3.5) / D + 1e-5


def test_surrnum_dismissal_rate_matches(draws):
    _, dismiss_p, wall_p = _expected(draws["x"], draws["surr"], draws["bpos"], draws["bnum"], draws["slot"])
    all_, prob = draws["cnt"][0], draws["cnt"][1]
    for n, k in ((all_, prob), (draws["used"], draws["o_dismissed"])):
        rate = k / n
        sd = np.sqrt(dismiss_p * (1 - dismiss_p) / n)
        assert abs(rate - dismiss_p) < 5 * sd
    # the proposals dismissed by the wall: all - prob-dismissed - NUM accepted
    wall = (all_ - prob - NUM) / all_
    assert abs(wall - wall_p) < 5 * np.sqrt(wall_p * (1 - wall_p) / all_)
