"""ifgf_mult_device_noalloc: the matvec for callers that cannot allocate
device memory when they apply the operator (inside a stream capture, or
under a memory pool that owns the GPU).  It must give the same result as
ifgf_mult_device, call after call, although every call reuses one fixed
64 MiB device scratch array that still holds the previous call's data.

Kept in its own file, collected last, so that a run stopping at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from ifgf_b200 import _lib
from ifgf_b200 import workloads as W

from .helpers import make_gpu_op, rel2

TOL = 1e-12


def _run(fn, op, w_dev, u_dev, stream):
    rc = fn(op._h, C.c_void_p(w_dev.data_ptr()), C.c_void_p(u_dev.data_ptr()),
            C.c_void_p(stream.cuda_stream))
    _lib.check(rc)


@pytest.mark.gpu
@pytest.mark.parametrize("name,k", [("helmholtz", 10.0), ("laplace", 0.0)])
def test_noalloc_matches_allocating_entry_point(name, k):
    import torch

    n = 3000
    pts = W.sphere_points(n, seed=0)
    op = make_gpu_op(name, leaf=50, order=8, k=k)
    op.init(pts, pts)
    dtype = torch.float64 if name == "laplace" else torch.complex128
    stream = torch.cuda.current_stream()
    for call, seed in enumerate((1, 5)):  # two calls in a row, different densities
        w = W.densities(n, complex_=(name != "laplace"), seed=seed)
        w_dev = torch.from_numpy(w).cuda()
        u_ref = torch.empty(n, dtype=dtype, device="cuda")
        u_new = torch.full((n,), float("nan"), dtype=dtype, device="cuda")
        _run(_lib.lib.ifgf_mult_device, op, w_dev, u_ref, stream)
        _run(_lib.lib.ifgf_mult_device_noalloc, op, w_dev, u_new, stream)
        torch.cuda.synchronize()
        a, b = u_new.cpu().numpy(), u_ref.cpu().numpy()
        assert np.all(np.isfinite(a)), call
        assert rel2(a, b) <= TOL, (call, rel2(a, b))


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
