"""Batched right-hand sides.

The mixed pipeline runs the right-hand sides in groups of four that share
the kernel and geometry evaluations, all groups (up to 64 right-hand sides)
in one launch per stage and level; every right-hand side must equal
its own single matvec (to FP32 rounding: the leaf factors are evaluated at
unit density and then scaled) and the FP64 pipeline within the mixed
tolerance.  The FP64 batch is the loop of single matvecs.
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W

from .helpers import densities_for, init_op, make_gpu_op, rel2

MIXED_TOL = 2e-5


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["helmholtz", "laplace", "modified_helmholtz", "combined_field"])
def test_batched_mixed_equals_single(name):
    n = 8000
    pts = W.sphere_points(n, seed=0)
    g = make_gpu_op(name, leaf=50, order=8)
    init_op(g, name, pts, pts)
    B = 6  # one full group of four and a padded group of two
    w = np.stack([densities_for(name, n, seed=10 + b) for b in range(B)])
    u64 = g.mult_batch(w)
    for b in range(B):
        assert rel2(u64[b], g.mult(w[b])) <= 1e-15
    g.set_precision("mixed")
    ub = g.mult_batch(w)
    for b in range(B):
        us = g.mult(w[b])
        assert rel2(ub[b], us) <= 1e-6, (b, rel2(ub[b], us))
        assert rel2(ub[b], u64[b]) <= MIXED_TOL
    assert g.stats()["missing_cone_lookups"] == 0


@pytest.mark.gpu
def test_batched_device_api_and_order_fallback():
    import torch

    n = 6000
    pts = W.sphere_points(n, seed=0)
    for order in (9, 11):  # fixed-order batched path; runtime-order fallback
        g = make_gpu_op("helmholtz", leaf=50, order=order)
        g.init(pts, pts)
        g.set_precision("mixed")
        w = np.stack([densities_for("helmholtz", n, seed=b) for b in range(5)])
        dw = torch.from_numpy(w).cuda()
        du = torch.empty_like(dw)
        g.mult_batch_device(dw.data_ptr(), du.data_ptr(), 5,
                            torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        u = du.cpu().numpy()
        for b in range(5):
            assert rel2(u[b], g.mult(w[b])) <= 1e-6


@pytest.mark.gpu
def test_plane_groups_in_one_launch_and_across_launches():
    # 70 right-hand sides: one launch of 64 planes (16 groups) and one of 6
    n = 4000
    pts = W.sphere_points(n, seed=0)
    g = make_gpu_op("helmholtz", leaf=50, order=8)
    g.init(pts, pts)
    g.set_precision("mixed")
    w = np.stack([densities_for("helmholtz", n, seed=100 + b) for b in range(70)])
    ub = g.mult_batch(w)
    for b in (0, 3, 4, 17, 63, 64, 69):
        assert rel2(ub[b], g.mult(w[b])) <= 1e-6, b


@pytest.mark.gpu
def test_batch_planes_follow_a_reinitialised_tree():
    # the plane buffers of a batch run before a re-init (finer cone grids,
    # larger planes) must not be reused at their old size
    n = 6000
    pts = W.sphere_points(n, seed=0)
    g = make_gpu_op("helmholtz", leaf=50, order=8, k=10.0)
    g.init(pts, pts)
    g.set_precision("mixed")
    w = np.stack([densities_for("helmholtz", n, seed=b) for b in range(5)])
    g.mult_batch(w)
    g.set_wavenumber(60.0)  # new grids: a full init
    fresh = make_gpu_op("helmholtz", leaf=50, order=8, k=60.0)
    fresh.init(pts, pts)
    fresh.set_precision("mixed")
    # the same upward kernel in both (each operator's autotuner times its own
    # launches and may pick the other kernel on a near tie)
    for path in ("ffma", "tensor"):
        g.set_upward_path(path)
        fresh.set_upward_path(path)
        ug, uf = g.mult_batch(w), fresh.mult_batch(w)
        for b in range(5):
            assert rel2(ug[b], uf[b]) <= 1e-14, (path, b)


@pytest.mark.gpu
def test_results_into_caller_arrays():
    # out= writes into the caller's (here pinned) arrays, as a new array would
    import torch

    n = 4000
    pts = W.sphere_points(n, seed=0)
    g = make_gpu_op("helmholtz", leaf=50, order=8)
    g.init(pts, pts)
    g.set_precision("mixed")
    w = np.stack([densities_for("helmholtz", n, seed=b) for b in range(6)])
    pinned = torch.empty((6, n), dtype=torch.complex128).pin_memory().numpy()
    assert g.mult_batch(w, out=pinned) is pinned
    assert np.array_equal(pinned, g.mult_batch(w))
    one = np.empty(n, dtype=np.complex128)
    assert g.mult(w[0], out=one) is one
    assert np.array_equal(one, g.mult(w[0]))
    with pytest.raises(ValueError):
        g.mult_batch(w, out=np.empty((6, n), dtype=np.complex64))


@pytest.mark.gpu
def test_pinned_host_batches_are_pipelined_and_equal():
    # pinned input and output: groups of four overlap their copies with the
    # matvecs of the neighbouring groups; the result is the same
    import torch

    n = 5000
    pts = W.sphere_points(n, seed=0)
    g = make_gpu_op("helmholtz", leaf=50, order=8)
    g.init(pts, pts)
    g.set_precision("mixed")
    w = np.stack([densities_for("helmholtz", n, seed=40 + b) for b in range(9)])
    ref = g.mult_batch(w)
    wp = torch.from_numpy(w).pin_memory().numpy()
    up = torch.empty((9, n), dtype=torch.complex128).pin_memory().numpy()
    for _ in range(2):
        g.mult_batch(wp, out=up)
        assert np.array_equal(up, ref)
