"""Frequency sets: one operator moved across wavenumbers with set_wavenumber.

The convolution-quadrature set of the batching workload uses the modified
Helmholtz kernel e^{-s r}/(4 pi r) at s_l = (1 - 0.5 z_l)/dt,
z_l = 0.9 e^{2 pi i l/64}, dt = 0.01.  Every frequency there gives the same
cone grids, so the operator keeps its tree and cone maps and only recomputes
the centre-shift factors; the result must equal a freshly built operator's
at that frequency.  A wavenumber that changes the grids re-initialises.
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W

from .helpers import rel2


def cq_wavenumbers(count=64, dt=0.01):
    z = 0.9 * np.exp(2j * np.pi * np.arange(count) / count)
    return (1.0 - 0.5 * z) / dt


@pytest.mark.gpu
def test_cq_frequency_set_reuses_tree_and_matches_fresh_operators():
    import ifgf_b200 as G

    n = 20000
    pts = W.sphere_points(n, seed=0)
    ks = cq_wavenumbers()[::8]
    op = G.ModifiedHelmholtzIfgfOperator(ks[0], 100, 8)
    op.init(pts, pts)
    grids = [op.grid(l, s).tolist() for l in range(op.levels()) for s in (0, 1)]
    idx = W.sample_targets(n, 200, seed=2)
    for l, k in enumerate(ks):
        w = W.densities(n, seed=10 + l)
        op.set_wavenumber(k)
        assert [op.grid(lv, s).tolist() for lv in range(op.levels()) for s in (0, 1)] == grids
        u = op.mult(w)
        fresh = G.ModifiedHelmholtzIfgfOperator(k, 100, 8)
        fresh.init(pts, pts)
        assert rel2(u, fresh.mult(w)) <= 1e-14, l
        d = op.direct_eval(w, idx)
        assert rel2(u[idx], d) <= 1e-4, (l, rel2(u[idx], d))


@pytest.mark.gpu
def test_wavenumber_change_with_new_grids_reinitialises():
    import ifgf_b200 as G

    n = 15000
    pts = W.sphere_points(n, seed=0)
    w = W.densities(n, seed=1)
    op = G.HelmholtzIfgfOperator(20.0, 64, 8)
    op.init(pts, pts)
    g20 = op.grid(2, 1).tolist()
    op.set_wavenumber(60.0)
    assert op.grid(2, 1).tolist() != g20  # kH/4 grew: finer cone grid
    fresh = G.HelmholtzIfgfOperator(60.0, 64, 8)
    fresh.init(pts, pts)
    assert rel2(op.mult(w), fresh.mult(w)) <= 1e-14
    # mixed precision and batched right-hand sides follow the new wavenumber
    op.set_precision("mixed")
    fresh.set_precision("mixed")
    wb = np.stack([w, W.densities(n, seed=2)])
    assert rel2(op.mult_batch(wb), fresh.mult_batch(wb)) <= 1e-14
