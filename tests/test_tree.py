"""Host octree and KIFMM interaction lists (no GPU needed).

The lists built in C++ (stkfmm_b200/csrc/stk_tree.cpp) are checked against
brute-force restatements of the KIFMM definitions over every node pair.
"""
import itertools

import numpy as np
import pytest

from helpers import clustered_points
from stkfmm_b200 import Octree


def boxes(t):
    h = 0.5 ** t.level.astype(np.float64)
    lo = t.ixyz * h[:, None]
    return lo, lo + h[:, None]


def shifts(pbc):
    rng = [(-1, 0, 1) if k < pbc else (0,) for k in range(3)]
    return list(itertools.product(*rng))


def code(s):
    return (s[0] + 1) + 3 * (s[1] + 1) + 9 * (s[2] + 1)


def adjacent(lo, hi, a, s, b):
    alo = lo[a] + np.array(s, dtype=np.float64)
    ahi = hi[a] + np.array(s, dtype=np.float64)
    return bool(np.all(alo <= hi[b]) and np.all(lo[b] <= ahi))


def to_sets(off, ent):
    return [set(int(e) for e in ent[off[i]:off[i + 1]]) for i in range(len(off) - 1)]


def brute_lists(t, src_count, trg_count, pbc):
    lo, hi = boxes(t)
    nn = t.num_nodes
    leaf = t.first_child < 0
    S = shifts(pbc)
    U = [set() for _ in range(nn)]
    W = [set() for _ in range(nn)]
    V = [set() for _ in range(nn)]
    X = [set() for _ in range(nn)]
    for b in range(nn):
        if trg_count[b] == 0:
            continue
        for a in range(nn):
            if src_count[a] == 0:
                continue
            for s in S:
                adj = adjacent(lo, hi, a, s, b)
                if leaf[b] and leaf[a] and adj:
                    U[b].add((a << 5) | code(s))
                pa = t.parent[a]
                pb = t.parent[b]
                if pa >= 0 and not adj:
                    if leaf[b] and t.level[a] > t.level[b] and adjacent(lo, hi, pa, s, b):
                        W[b].add((a << 5) | code(s))
                    if pb >= 0 and t.level[a] == t.level[b] and adjacent(lo, hi, pa, s, pb):
                        V[b].add((a << 5) | code(s))
                # X: b is in the W relation of the source leaf a (a need not hold targets)
                if pb >= 0 and not adj and leaf[a] and t.level[b] > t.level[a] and adjacent(lo, hi, a, s, pb):
                    X[b].add((a << 5) | code(s))
    return U, V, W, X


CASES = [
    ("uniform", 0, 16),
    ("clustered", 0, 12),
    ("uniform", 3, 16),
    ("clustered", 2, 10),
    ("clustered", 1, 10),
    ("clustered-apart", 0, 12),  # targets apart from the sources: leaves with sources only
    ("clustered-apart", 3, 12),
]


@pytest.mark.parametrize("dist,pbc,max_pts", CASES)
def test_lists_match_kifmm_definitions(dist, pbc, max_pts):
    rng = np.random.default_rng(7 + pbc)
    n = 700
    pts = rng.random((n, 3)) if dist == "uniform" else clustered_points(rng, n, nclusters=4, sigma=0.05)
    trg = rng.random((n // 2, 3)) if dist == "clustered-apart" else pts[: n // 2]
    t = Octree(pts, max_pts, pbc, sl=pts, trg=trg)
    _, sb, se = t.point_set(0)
    _, tb, te = t.point_set(2)
    src_count = se - sb
    trg_count = te - tb
    U, V, W, X = brute_lists(t, src_count, trg_count, pbc)
    for name, ref in zip("UVWX", (U, V, W, X)):
        got = to_sets(*t.list(name))
        bad = [i for i in range(t.num_nodes) if got[i] != ref[i]]
        assert not bad, (name, bad[:5], [sorted(got[i]) for i in bad[:1]], [sorted(ref[i]) for i in bad[:1]])


@pytest.mark.parametrize("pbc", [0, 3])
def test_tree_invariants(pbc):
    rng = np.random.default_rng(3)
    pts = clustered_points(rng, 5000, nclusters=6, sigma=0.01)
    sl = pts
    dl = rng.random((300, 3))
    t = Octree(pts, 40, pbc, sl=sl, dl=dl, trg=pts)
    leaf = t.first_child < 0
    for k, P in enumerate((sl, dl, pts)):
        perm, b, e = t.point_set(k)
        assert sorted(perm.tolist()) == list(range(len(P)))
        # every point lies inside the leaf that owns it
        lo, hi = boxes(t)
        for i in np.flatnonzero(leaf):
            q = P[perm[b[i]:e[i]]]
            assert np.all(q >= lo[i]) and np.all(q < hi[i])
        # leaves partition each set; children partition their parent
        assert (e - b)[leaf].sum() == len(P)
        for i in np.flatnonzero(~leaf):
            c = t.first_child[i]
            assert b[c] == b[i] and e[c + 7] == e[i]
            assert np.all(e[c:c + 7] == b[c + 1:c + 8])
    # leaves hold at most max_pts tree points unless refinement stopped at max depth
    _, b, e = t.point_set(2)
    assert np.all(((e - b)[leaf] <= 40) | (t.level[leaf] >= 20))


def test_ulist_symmetric_when_sources_are_targets():
    rng = np.random.default_rng(11)
    pts = clustered_points(rng, 3000, nclusters=5, sigma=0.03)
    t = Octree(pts, 32, 0, sl=pts, trg=pts)
    U = to_sets(*t.list("U"))
    for b, s in enumerate(U):
        for e in s:
            a, c = e >> 5, e & 31
            assert ((b << 5) | (26 - c)) in U[a]


def test_all_coincident_points_stop_at_max_depth():
    pts = np.full((50, 3), 0.3)
    t = Octree(pts, 4, 0, sl=pts, trg=pts)
    assert t.depth == 20
    off, ent = t.list("U")
    # the single non-empty leaf sees itself
    nonempty = [i for i in range(t.num_nodes) if off[i + 1] > off[i]]
    assert len(nonempty) == 1 and (ent[off[nonempty[0]]] >> 5) == nonempty[0]


def test_out_of_box_rejected():
    pts = np.array([[0.5, 0.5, 1.0]])
    with pytest.raises(Exception):
        Octree(pts, 4, 0, sl=pts, trg=pts)


def test_empty_sets():
    pts = np.random.default_rng(0).random((100, 3))
    t = Octree(pts, 8, 0, sl=np.zeros((0, 3)), trg=pts)
    off, ent = t.list("U")
    assert len(ent) == 0
