"""ifgf_mult_device_noalloc: the matvec for callers that cannot allocate
device memory when they apply the operator -- an application whose own
memory pool has reserved the whole GPU, or a real-time loop that must not
stall on cudaMalloc's implicit synchronisation.  It must give the same
result as ifgf_mult_device, call after call, although every call reuses one
fixed 64 MiB device scratch array that still holds the previous call's data
(possibly another operator's).

Kept in its own file, collected last, so that a run stopping at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from ifgf_b200 import _lib
from ifgf_b200 import workloads as W

from .helpers import make_gpu_op, rel2

# same kernels on the same inputs as ifgf_mult_device: FP64 to the parity
# tolerance, the mixed pipeline to FP32 rounding
TOL = {"fp64": 1e-12, "mixed": 1e-6}


def _run(fn, op, w_dev, u_dev, stream):
    rc = fn(op._h, C.c_void_p(w_dev.data_ptr()), C.c_void_p(u_dev.data_ptr()),
            C.c_void_p(stream.cuda_stream))
    _lib.check(rc)


def _compare(op, n, complex_, seed, precision):
    import torch

    dtype = torch.complex128 if complex_ else torch.float64
    stream = torch.cuda.current_stream()
    w = W.densities(n, complex_=complex_, seed=seed)
    w_dev = torch.from_numpy(w).cuda()
    u_ref = torch.empty(n, dtype=dtype, device="cuda")
    u_new = torch.full((n,), float("nan"), dtype=dtype, device="cuda")
    _run(_lib.lib.ifgf_mult_device, op, w_dev, u_ref, stream)
    _run(_lib.lib.ifgf_mult_device_noalloc, op, w_dev, u_new, stream)
    torch.cuda.synchronize()
    a, b = u_new.cpu().numpy(), u_ref.cpu().numpy()
    assert np.all(np.isfinite(a))
    return rel2(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,k", [("helmholtz", 10.0), ("laplace", 0.0)])
def test_noalloc_matches_allocating_entry_point(name, k, precision):
    n = 3000
    pts = W.sphere_points(n, seed=0)
    op = make_gpu_op(name, leaf=50, order=8, k=k)
    op.init(pts, pts)
    op.set_precision(precision)
    for call, seed in enumerate((1, 5)):  # two calls in a row, different densities
        err = _compare(op, n, name != "laplace", seed, precision)
        assert err <= TOL[precision], (call, err)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_two_operators_interleaved(precision):
    """Operator A, then a larger operator B with other points and more fine
    coefficients, then A again: each call starts from the other operator's
    leftovers in the shared array."""
    na, nb = 3000, 4000
    pa = W.sphere_points(na, seed=0)
    pb = W.ellipsoid_points(nb, seed=3)
    opa = make_gpu_op("helmholtz", leaf=50, order=8, k=10.0)
    opa.init(pa, pa)
    opb = make_gpu_op("helmholtz", leaf=50, order=8, k=16.0)
    opb.init(pb, pb)
    assert opb.stats()["fine_cones_total"] > opa.stats()["fine_cones_total"]
    for op in (opa, opb):
        op.set_precision(precision)
    for call, (op, n, seed) in enumerate(((opa, na, 1), (opb, nb, 2), (opa, na, 3))):
        err = _compare(op, n, True, seed, precision)
        assert err <= TOL[precision], (call, err)


@pytest.mark.gpu
def test_noalloc_rejects_problems_beyond_the_fixed_scratch():
    import torch

    n = 60000
    pts = W.sphere_points(n, seed=0)
    op = make_gpu_op("helmholtz", leaf=50, order=10, k=80.0)
    op.init(pts, pts)
    w_dev = torch.from_numpy(W.densities(n, seed=1)).cuda()
    u_dev = torch.empty_like(w_dev)
    rc = _lib.lib.ifgf_mult_device_noalloc(op._h, C.c_void_p(w_dev.data_ptr()),
                                           C.c_void_p(u_dev.data_ptr()), None)
    assert rc == 1
    assert "no-allocation scratch" in _lib.lib.ifgf_last_error().decode()
