"""The octree built on the GPU equals the host builder's bit for bit.

The host builder (plan-only init, no GPU) is checked against the oracle's
restatement of octree.hpp in test_planner.py; here the GPU build of a
regular init must give the same Morton permutation, the same boxes (ranges,
parents, children, leaf flags) and the same bounding boxes at every level,
including point sets with exact duplicates, a flat (degenerate) dimension
and leaves smaller than a warp.
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W


def _sets():
    rng = np.random.default_rng(7)
    dup = W.sphere_points(20000, seed=0)
    dup[:, 10000:12000] = dup[:, :2000]  # exact duplicates
    flat = rng.standard_normal((3, 30000))
    flat[2] = 0.0  # all points in the plane z = 0
    return [
        ("sphere", W.sphere_points(40000, seed=0), 100),
        ("ellipsoid", W.ellipsoid_points(60000, seed=0), 64),
        ("duplicates", dup, 50),
        ("flat", flat, 30),
        ("cube_small_leaves", rng.uniform(-1, 1, (3, 20000)), 7),
        ("tiny", rng.uniform(-1, 1, (3, 40)), 100),
    ]


@pytest.mark.gpu
@pytest.mark.parametrize("name,pts,leaf", _sets(), ids=lambda v: v if isinstance(v, str) else "")
def test_gpu_octree_equals_host_octree(name, pts, leaf):
    import ifgf_b200 as G

    tg = W.sphere_points(5000, seed=3) * 1.5
    gpu = G.HelmholtzIfgfOperator(5.0, leaf, 8)
    gpu.init(pts, tg)
    host = G.HelmholtzIfgfOperator(5.0, leaf, 8)
    host.init_plan_only(pts, tg)
    for which in (0, 1):
        assert np.array_equal(gpu.permutation(which), host.permutation(which)), which
        assert gpu.levels(which) == host.levels(which)
        for lvl in range(host.levels(which)):
            gi, gb = gpu.boxes(lvl, which)
            hi, hb = host.boxes(lvl, which)
            assert np.array_equal(gi, hi), (which, lvl)
            assert np.array_equal(gb, hb), (which, lvl)
    st = gpu.stats()
    assert st["init_tree_ms"] >= 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("name,pts,leaf", _sets(), ids=lambda v: v if isinstance(v, str) else "")
def test_gpu_interaction_lists_equal_host_lists(name, pts, leaf):
    """The dual-tree walk on the GPU gives every source box the host walker's
    far and near lists, in the same (discovery) order, and the same pair
    counts."""
    import ifgf_b200 as G

    tg = W.sphere_points(5000, seed=3) * 1.5
    gpu = G.HelmholtzIfgfOperator(5.0, leaf, 8)
    gpu.init(pts, tg)
    host = G.HelmholtzIfgfOperator(5.0, leaf, 8)
    host.init_plan_only(pts, tg)
    sg, sh = gpu.stats(), host.stats()
    for key in ("near_pairs", "far_pairs", "near_point_pairs", "far_target_evals",
                "far_point_pairs", "target_leaf_far_evals", "target_leaf_far_point_pairs",
                "target_leaf_near_point_pairs"):
        assert sg[key] == sh[key], key
    assert sg["target_leaf_far_evals"] == sg["far_target_evals"]
    assert sg["target_leaf_far_point_pairs"] == sg["far_point_pairs"]
    assert sg["target_leaf_near_point_pairs"] == sg["near_point_pairs"]
    for lvl in range(host.levels(0)):
        for box in range(host.num_boxes(lvl, 0)):
            for far in (0, 1):
                a = gpu.interaction_list(lvl, box, far)
                b = host.interaction_list(lvl, box, far)
                assert np.array_equal(a, b), (lvl, box, far)


_TL_KEYS = ("target_leaf_far_evals", "target_leaf_far_point_pairs",
            "target_leaf_near_point_pairs", "target_leaf_lists_checksum", "target_leaves")


@pytest.mark.gpu
@pytest.mark.parametrize("name,pts,leaf", _sets(), ids=lambda v: v if isinstance(v, str) else "")
def test_gpu_target_leaf_lists_equal_host_lists(name, pts, leaf):
    """The target-leaf lists built on the GPU (stable radix sort by target,
    ancestor concatenation, one warp per leaf) equal the host build entry for
    entry: the same work sums and the same position-weighted checksum."""
    import ifgf_b200 as G

    for tg in (None, W.sphere_points(5000, seed=3) * 1.5):
        t = pts if tg is None else tg
        gpu = G.HelmholtzIfgfOperator(5.0, leaf, 8)
        gpu.init(pts, t)
        host = G.HelmholtzIfgfOperator(5.0, leaf, 8)
        host.init_plan_only(pts, t)
        sg, sh = gpu.stats(), host.stats()
        for key in _TL_KEYS[:4]:
            assert sg[key] == sh[key], (key, tg is None)
        assert sg["target_leaf_far_evals"] == sg["far_target_evals"]
        assert sg["target_leaf_near_point_pairs"] == sg["near_point_pairs"]


@pytest.mark.gpu
def test_gpu_target_leaf_lists_sharded_and_host_walk():
    """Per-rank lists of a sharded operator (another rank's source boxes
    dropped) and lists from pairs uploaded after a host walk (a cutoff
    predicate) equal the host build."""
    import ifgf_b200 as G

    pts = W.ellipsoid_points(60000, seed=0)
    tot = None
    sums = [0, 0, 0]
    for rank in range(3):
        gpu = G.HelmholtzIfgfOperator(20.0, 60, 8)
        gpu.set_shard(rank, 3)
        gpu.init(pts, pts)
        host = G.HelmholtzIfgfOperator(20.0, 60, 8)
        host.set_shard(rank, 3)
        host.init_plan_only(pts, pts)
        sg, sh = gpu.stats(), host.stats()
        for key in _TL_KEYS[:4]:
            assert sg[key] == sh[key], (key, rank)
        for i, key in enumerate(_TL_KEYS[:3]):
            sums[i] += sg[key]
        tot = sg
    assert sums == [tot["far_target_evals"], tot["far_point_pairs"], tot["near_point_pairs"]]

    def cut(d):
        return d > 0.3

    gpu = G.HelmholtzIfgfOperator(20.0, 60, 8)
    gpu.init(pts, pts, cutOff=cut)
    host = G.HelmholtzIfgfOperator(20.0, 60, 8)
    host.init_plan_only(pts, pts, cutOff=cut)
    sg, sh = gpu.stats(), host.stats()
    assert sg["dropped_pairs"] > 0
    for key in _TL_KEYS[:4]:
        assert sg[key] == sh[key], key
