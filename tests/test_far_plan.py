"""The far-field plan of the batched mixed matvecs (ifgf_set_far_plan): the
cone lookups of every (target, far box) pair done once and stored grouped
and sorted by cone, against the far kernel that does them in every matvec
(evaluateFromInterp, ifgfoperator.hpp:1736-1891).  The plan holds the same
records the on-the-fly kernel builds and each owner adds its pairs in the
same order, so the results are equal bit for bit.
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W

from .helpers import KERNELS, densities_for, init_op, make_gpu_op, rel2


def _on_off(op, fn):
    """fn() without the plan, then with it (the plan stays built)."""
    out = {}
    for on in (False, True):
        op.set_far_plan(on)
        out[on] = fn()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(KERNELS))
def test_far_plan_equals_on_the_fly_all_kernels(name):
    n = 12000
    pts = W.ellipsoid_points(n, seed=0)
    g = make_gpu_op(name, leaf=50, order=8)
    init_op(g, name, pts, pts)
    g.set_precision("mixed")
    wb = np.stack([densities_for(name, n) * (1.0 + 0.1 * b) for b in range(5)])
    u = _on_off(g, lambda: g.mult_batch(wb))
    assert np.array_equal(u[True], u[False]), name
    st = g.stats()["far_plan"]
    assert st["built"] == 1 and st["records"] > 0 and st["bytes"] > 0
    assert g.stats()["missing_cone_lookups"] == 0


@pytest.mark.gpu
def test_far_plan_multi_wavenumber_and_memory_release():
    import ifgf_b200 as G

    from .test_frequency import cq_wavenumbers

    n = 15000
    pts = W.sphere_points(n, seed=0)
    ks = cq_wavenumbers()[:12]
    w = np.stack([W.densities(n, seed=10 + l) for l in range(len(ks))])
    op = G.ModifiedHelmholtzIfgfOperator(ks[0], 100, 8)
    op.init(pts, pts)
    op.set_precision("mixed")
    u = _on_off(op, lambda: op.mult_wavenumbers(ks, w))
    assert np.array_equal(u[True], u[False])
    op.set_far_plan(False)
    st = op.stats()["far_plan"]
    assert st["on"] == 0 and st["built"] == 0 and st["bytes"] == 0


@pytest.mark.gpu
def test_far_plan_leaves_larger_than_a_block_and_sharded():
    """Leaves of up to 400 targets (several 256-target chunks per leaf) and
    a sharded operator (a rank's far lists hold only its source boxes)."""
    import ifgf_b200 as G

    n = 20000
    pts = W.ellipsoid_points(n, seed=3)
    wb = np.stack([W.densities(n, seed=20 + b) for b in range(4)])
    g = G.HelmholtzIfgfOperator(30.0, 400, 8)
    g.init(pts, pts)
    g.set_precision("mixed")
    u = _on_off(g, lambda: g.mult_batch(wb))
    assert np.array_equal(u[True], u[False])
    assert g.stats()["far_plan"]["chunks"] > g.stats()["target_leaves"]
    parts = []
    for rank in range(2):
        s = G.HelmholtzIfgfOperator(30.0, 60, 8)
        s.set_shard(rank, 2)
        s.init(pts, pts)
        s.set_precision("mixed")
        us = _on_off(s, lambda: s.mult_batch(wb))
        assert np.array_equal(us[True], us[False]), rank
        parts.append(us[True])
    full = G.HelmholtzIfgfOperator(30.0, 60, 8)
    full.init(pts, pts)
    full.set_precision("mixed")
    assert rel2(parts[0] + parts[1], full.mult_batch(wb)) <= 2e-6


@pytest.mark.gpu
def test_far_plan_rebuilt_after_reinit():
    """A second init (other points) drops the plan of the first; the next
    batched matvec builds the plan of the new tables."""
    import ifgf_b200 as G

    g = G.HelmholtzIfgfOperator(20.0, 60, 8)
    g.set_precision("mixed")
    for seed in (0, 1):
        n = 8000 + 2000 * seed
        pts = W.ellipsoid_points(n, seed=seed)
        g.init(pts, pts)
        assert g.stats()["far_plan"]["built"] == 0
        wb = np.stack([W.densities(n, seed=5 + b) for b in range(3)])
        u = _on_off(g, lambda: g.mult_batch(wb))
        assert np.array_equal(u[True], u[False]), seed


@pytest.mark.gpu
@pytest.mark.parametrize("order", [9, 10])
def test_far_plan_higher_orders(order):
    """Orders 9 and 10 (low-order cones (3,6,6) and (4,7,7): larger slots,
    other slot counts and CTAs per SM): the plan equals the no-plan kernel
    bit for bit, and the batched mixed matvec stays within the mixed
    tolerance of the FP64 pipeline."""
    import ifgf_b200 as G

    n = 15000
    pts = W.ellipsoid_points(n, seed=1)
    g = G.HelmholtzIfgfOperator(40.0, 60, order)
    g.init(pts, pts)
    wb = np.stack([W.densities(n, seed=30 + b) for b in range(4)])
    u64 = np.stack([g.mult(w) for w in wb])
    g.set_precision("mixed")
    u = _on_off(g, lambda: g.mult_batch(wb))
    assert np.array_equal(u[True], u[False]), order
    assert rel2(u[True], u64) <= 2e-5, rel2(u[True], u64)
    assert g.stats()["far_plan"]["slots_per_group"] in (16, 24)
