"""The wavenumber derivative (dA/dk) w of the Helmholtz and combined-field
kernels.

There is no reference counterpart: the derivative kernels are checked
against central finite differences (h = 1e-6) of the reference kernels'
FP64 direct sums, the oracle's IFGF approximation of the derivative against
its direct sum, and the CUDA path against the oracle (<= 1e-12, the parity
bar of every kernel).
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W
from oracle import oracle as O

from .helpers import densities_for, make_gpu_op, make_oracle_op, rel2

FD_H = 1e-6
CASES = [("helmholtz", "helmholtz_dk", False), ("combined_field", "combined_field_dk", True)]


def _init(op, pts, normals):
    if normals:
        op.init(pts, pts, pts)
    else:
        op.init(pts, pts)


@pytest.mark.parametrize("base,dk,normals", CASES)
def test_oracle_dk_kernel_is_the_k_derivative(base, dk, normals):
    n = 1500
    pts = W.sphere_points(n, seed=0)
    w = densities_for(base, n)
    idx = np.arange(0, n, 11)
    nrm = pts if normals else None
    k = 20.0
    up = O.direct_sum(base, k + FD_H, pts, w, pts, idx, normals=nrm)
    um = O.direct_sum(base, k - FD_H, pts, w, pts, idx, normals=nrm)
    d = O.direct_sum(dk, k, pts, w, pts, idx, normals=nrm)
    assert rel2((up - um) / (2 * FD_H), d) <= 1e-8


@pytest.mark.parametrize("base,dk,normals", CASES)
def test_oracle_dk_ifgf_converges(base, dk, normals):
    n = 2500
    pts = W.sphere_points(n, seed=0)
    w = densities_for(base, n)
    idx = np.arange(0, n, 13)
    k = 20.0
    d = O.direct_sum(dk, k, pts, w, pts, idx, normals=pts if normals else None)
    errs = []
    for p in (8, 10):
        op = O.OracleOperator(dk, k, 100, p)
        _init(op, pts, normals)
        errs.append(rel2(op.mult(w)[idx], d))
    assert errs[0] < 1e-3 and errs[1] < 1e-6, errs


@pytest.mark.gpu
@pytest.mark.parametrize("base,dk,normals", CASES)
def test_dk_parity_with_oracle(base, dk, normals):
    n = 6000
    pts = W.sphere_points(n, seed=0)
    w = densities_for(base, n)
    g = make_gpu_op(base, leaf=50, order=8)
    _init(g, pts, normals)
    o = O.OracleOperator(dk, 20.0, 50, 8)
    _init(o, pts, normals)
    ug = g.mult_dk(w)
    uo = o.mult(w)
    assert rel2(ug, uo) <= 1e-12, rel2(ug, uo)
    # the base matvec is untouched by the derivative's tables
    ob = make_oracle_op(base, leaf=50, order=8)
    _init(ob, pts, normals)
    assert rel2(g.mult(w), ob.mult(w)) <= 1e-12
    assert g.stats()["missing_cone_lookups"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("base,dk,normals", CASES)
def test_dk_against_finite_differences_and_direct(base, dk, normals):
    n = 8000
    pts = W.sphere_points(n, seed=0)
    w = densities_for(base, n)
    idx = W.sample_targets(n, 300, seed=2)
    k = 20.0
    g = make_gpu_op(base, leaf=64, order=10, k=k)
    _init(g, pts, normals)
    d = g.direct_eval(w, idx, dk=True)
    gp = make_gpu_op(base, leaf=64, order=10, k=k + FD_H)
    gm = make_gpu_op(base, leaf=64, order=10, k=k - FD_H)
    _init(gp, pts, normals)
    _init(gm, pts, normals)
    fd = (gp.direct_eval(w, idx) - gm.direct_eval(w, idx)) / (2 * FD_H)
    assert rel2(fd, d) <= 1e-7
    u = g.mult_dk(w)
    assert rel2(u[idx], d) <= 1e-6, rel2(u[idx], d)
    # batched host call = one call per right-hand side
    w2 = np.stack([w, densities_for(base, n, seed=5)])
    u2 = g.mult_dk(w2)
    assert rel2(u2[0], u) <= 1e-15
    # mixed precision of the derivative
    g.set_precision("mixed")
    assert rel2(g.mult_dk(w), u) <= 5e-5


@pytest.mark.gpu
def test_dk_rejected_for_kernels_without_derivative():
    from ifgf_b200 import IfgfError

    n = 500
    pts = W.sphere_points(n, seed=0)
    g = make_gpu_op("laplace", leaf=50, order=8)
    g.init(pts, pts)
    with pytest.raises(IfgfError):
        g.mult_dk(np.ones(n))
