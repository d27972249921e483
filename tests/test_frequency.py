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
    # mixed precision and batched right-hand sides follow the new wavenumber,
    # on either upward kernel (pinned: the autotuner of each operator times
    # its own launches, and two near-equal timings may pick different
    # kernels, whose FP32 results differ in rounding)
    op.set_precision("mixed")
    fresh.set_precision("mixed")
    wb = np.stack([w, W.densities(n, seed=2)])
    for path in ("ffma", "tensor"):
        op.set_upward_path(path)
        fresh.set_upward_path(path)
        assert rel2(op.mult_batch(wb), fresh.mult_batch(wb)) <= 1e-14, path


@pytest.mark.gpu
def test_cq_set_in_one_multi_wavenumber_batch():
    """All 64 CQ frequencies in one pass (one launch per stage and level):
    each plane equals the operator moved to that frequency, and the FP64
    direct sum within the mixed tolerance."""
    import ifgf_b200 as G

    n = 20000
    pts = W.sphere_points(n, seed=0)
    ks = cq_wavenumbers()
    w = np.stack([W.densities(n, seed=10 + l) for l in range(len(ks))])
    op = G.ModifiedHelmholtzIfgfOperator(ks[0], 100, 8)
    op.init(pts, pts)
    op.set_precision("mixed")
    u = op.mult_wavenumbers(ks, w)
    assert op.stats()["missing_cone_lookups"] == 0
    ref = G.ModifiedHelmholtzIfgfOperator(ks[0], 100, 8)
    ref.init(pts, pts)
    ref.set_precision("mixed")
    idx = W.sample_targets(n, 200, seed=2)
    for l in range(0, len(ks), 7):
        ref.set_wavenumber(ks[l])
        # the planes form the centre-shift factor from tabulated distances,
        # the single matvec reads it tabulated: FP32 rounding apart
        assert rel2(u[l], ref.mult(w[l])) <= 2e-5, l
        d = ref.direct_eval(w[l], idx)
        assert rel2(u[l][idx], d) <= 1e-4, (l, rel2(u[l][idx], d))


@pytest.mark.gpu
def test_multi_wavenumber_helmholtz_band_and_fp64_loop():
    import ifgf_b200 as G

    n = 12000
    pts = W.sphere_points(n, seed=0)
    ks = 20.2 + 0.1 * np.arange(8)  # ceil(k H / 4) is the same at every level
    w = np.stack([W.densities(n, seed=20 + l) for l in range(len(ks))])
    op = G.HelmholtzIfgfOperator(20.5, 64, 8)
    op.init(pts, pts)
    grids = [op.grid(l, s).tolist() for l in range(op.levels()) for s in (0, 1)]
    u0 = op.mult(w[0])
    # FP64: the set_wavenumber loop, and the operator keeps its wavenumber
    u64 = op.mult_wavenumbers(ks, w)
    assert rel2(op.mult(w[0]), u0) <= 1e-15
    op.set_precision("mixed")
    umx = op.mult_wavenumbers(ks, w)
    for l, k in enumerate(ks):
        fresh = G.HelmholtzIfgfOperator(k, 64, 8)
        fresh.init(pts, pts)
        assert [fresh.grid(lv, s).tolist() for lv in range(fresh.levels()) for s in (0, 1)] == grids
        assert rel2(u64[l], fresh.mult(w[l])) <= 1e-14, l
        assert rel2(umx[l], u64[l]) <= 2e-5, (l, rel2(umx[l], u64[l]))


@pytest.mark.gpu
def test_multi_wavenumber_rejects_other_cone_grids():
    import ifgf_b200 as G

    n = 5000
    pts = W.sphere_points(n, seed=0)
    op = G.HelmholtzIfgfOperator(20.5, 64, 8)
    op.init(pts, pts)
    op.set_precision("mixed")
    w = np.stack([W.densities(n, seed=1)] * 2)
    with pytest.raises(Exception, match="cone grids"):
        op.mult_wavenumbers([20.5, 60.0], w)


@pytest.mark.gpu
def test_multi_wavenumber_device_entry_point():
    # device buffers on a torch stream give the host-buffer call's result
    import torch

    import ifgf_b200 as G

    n = 8000
    pts = W.sphere_points(n, seed=0)
    ks = cq_wavenumbers()[:6]
    w = np.stack([W.densities(n, seed=30 + l) for l in range(len(ks))])
    op = G.ModifiedHelmholtzIfgfOperator(ks[0], 100, 8)
    op.init(pts, pts)
    op.set_precision("mixed")
    uh = op.mult_wavenumbers(ks, w)
    dw = torch.from_numpy(w).cuda()
    du = torch.empty_like(dw)
    op.mult_wavenumbers_device(ks, dw.data_ptr(), du.data_ptr(),
                               torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ud = du.cpu().numpy()
    for l in range(len(ks)):
        assert rel2(ud[l], uh[l]) <= 1e-14, l
