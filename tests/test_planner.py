"""The product's host planner against the oracle's octree: Morton permutation,
box ranges and bounding boxes per level (octree.hpp:202-238, 1106-1184) and
the dual-tree interaction lists in discovery order (octree.hpp:255-349),
bit-exact.  Runs without a GPU (plan-only init)."""
import numpy as np
import pytest

import ifgf_b200 as G
from ifgf_b200 import workloads as W
from oracle import oracle as O


def _compare(src, tgt, leaf=100, cutoff=None):
    o = O.OracleOperator("laplace", 0, leaf, 8)
    o.init(src, tgt)
    g = G.LaplaceIfgfOperator(leaf, 8)
    g.init_plan_only(src, tgt, cutoff)
    for which, pts in ((0, src), (1, tgt)):
        assert g.levels(which) == o.levels(which)
        pg, po = g.permutation(which), o.perm(which)
        # identical up to the order of exactly coincident points, which the
        # reference's (unstable) std::sort leaves unspecified
        assert np.array_equal(pts[:, pg], pts[:, po])
        assert np.array_equal(np.sort(pg), np.arange(pts.shape[1]))
        for lvl in range(o.levels(which)):
            a, b = o.boxes(lvl, which)
            c, d = g.boxes(lvl, which)
            assert np.array_equal(a, c), (which, lvl)
            assert np.array_equal(b, d), (which, lvl)
    if cutoff is None:
        for lvl in range(o.levels()):
            for b in range(o.num_boxes(lvl)):
                for far in (0, 1):
                    assert np.array_equal(o.interaction_list(lvl, b, far),
                                          g.interaction_list(lvl, b, far)), (lvl, b, far)
    return g


@pytest.mark.parametrize("n", [1, 7, 100, 101, 2500, 20000])
def test_sphere(n):
    p = W.sphere_points(n, seed=0)
    _compare(p, p)


def test_ellipsoid_1e5():
    p = W.ellipsoid_points(100000, seed=0)
    _compare(p, p)


def test_different_sets_and_leaf_sizes():
    src = W.sphere_points(7000, seed=3)
    tgt = W.ellipsoid_points(4000, axes=(1.5, 0.7, 1.1), seed=9)
    for leaf in (1, 10, 64, 300):
        _compare(src, tgt, leaf)


def test_clustered_and_degenerate_points():
    rng = np.random.default_rng(5)
    # clusters, a plane (zero extent in z), exact duplicates, points on box mid-planes
    a = rng.normal(size=(3, 3000)) * 1e-3 + np.array([[0.3], [0.1], [-0.2]])
    b = rng.uniform(-1, 1, size=(3, 2000))
    b[2] = 0.25
    c = np.repeat(rng.uniform(-1, 1, size=(3, 50)), 4, axis=1)
    d = rng.uniform(-1, 1, size=(3, 500))
    d[0] = 0.0
    p = np.concatenate([a, b, c, d], axis=1)
    _compare(p, p, leaf=20)


def test_cutoff_predicate_drops_far_pairs():
    p = W.sphere_points(20000, seed=0)
    g0 = G.LaplaceIfgfOperator(100, 8)
    g0.init_plan_only(p, p)
    g1 = G.LaplaceIfgfOperator(100, 8)
    g1.init_plan_only(p, p, cutOff=lambda dist: dist > 1.0)
    s0 = [len(g0.interaction_list(l, b, 1)) for l in range(g0.levels()) for b in range(g0.num_boxes(l))]
    s1 = [len(g1.interaction_list(l, b, 1)) for l in range(g1.levels()) for b in range(g1.num_boxes(l))]
    assert sum(s1) < sum(s0)


def test_product_connectivity():
    n = 3000
    src = W.sphere_points(n, seed=0)
    tgt = W.sphere_points(2000, seed=8) * 1.05
    g = G.LaplaceIfgfOperator(30, 8)
    g.init_plan_only(src, tgt)
    cov = np.zeros((n, 2000), dtype=np.int32)
    for lvl in range(g.levels()):
        ints, _ = g.boxes(lvl)
        for b in range(len(ints)):
            s0, s1 = ints[b, 0], ints[b, 1]
            for far in (0, 1):
                for t0, t1 in g.interaction_list(lvl, b, far):
                    cov[s0:s1, t0:t1] += 1
    assert cov.min() == 1 and cov.max() == 1


def test_morton_order_matches_comparator():
    """Sorted neighbours of the product permutation are in the oracle's
    zorder_knn::Less order (zorder_less.hpp:212-248)."""
    p = W.ellipsoid_points(5000, seed=11)
    g = G.LaplaceIfgfOperator(100, 8)
    g.init_plan_only(p, p)
    perm = g.permutation(0)
    _, bb = g.boxes(0)
    mn, mx = bb[0, :3], bb[0, 3:]
    for i in range(len(perm) - 1):
        assert O.morton_less(mn, mx, p[:, perm[i]], p[:, perm[i + 1]])


@pytest.mark.parametrize("case", ["same", "distinct", "leaf_7", "cutoff"])
def test_target_leaf_lists_cover_every_pair(case):
    """The per-target-leaf CSR (a leaf's far list = its own far sources and
    every ancestor's) describes exactly the walk's work: each far pair (s, t)
    reaches the points of t through the leaves that partition t, each near
    pair once; weighting every entry by its source box's points checks the
    entries themselves, not only the list lengths.  Sharded, the ranks' lists
    add up to the same totals."""
    n = 60000
    src = W.ellipsoid_points(n, seed=0)
    tgt = src if case != "distinct" else W.sphere_points(n // 2, seed=3)
    leaf = 7 if case == "leaf_7" else 100
    # a cutoff drops the far pairs beyond distance 1.2 from the walk, and so
    # from the target-leaf lists
    cut = (lambda d: d > 1.2) if case == "cutoff" else None
    g = G.HelmholtzIfgfOperator(20.0, leaf, 6)
    g.init_plan_only(src, tgt, cut)
    st = g.stats()
    if cut is not None:
        assert st["dropped_pairs"] > 0
    assert st["target_leaf_far_evals"] == st["far_target_evals"] > 0
    assert st["target_leaf_far_point_pairs"] == st["far_point_pairs"] > 0
    assert st["target_leaf_near_point_pairs"] == st["near_point_pairs"] > 0
    far = farp = near = 0
    for rank in range(3):
        s = G.HelmholtzIfgfOperator(20.0, leaf, 6)
        s.set_shard(rank, 3)
        s.init_plan_only(src, tgt, cut)
        ss = s.stats()
        far += ss["target_leaf_far_evals"]
        farp += ss["target_leaf_far_point_pairs"]
        near += ss["target_leaf_near_point_pairs"]
    assert (far, farp, near) == (st["far_target_evals"], st["far_point_pairs"],
                                 st["near_point_pairs"])
