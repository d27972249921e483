"""The adjoint matvec A^H w.

The reference has no adjoint: the oracle for it is the reference's own
operators with the roles of sources and targets exchanged, composed as the
library composes them, and the dense kernel matrix of the oracle (A^H = its
conjugate transpose) at sizes where it fits in memory.  The CPU tests check
the kernel identities the composition rests on.
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W
from oracle import oracle as O

from .helpers import KERNELS, densities_for, make_gpu_op, make_oracle_op, rel2

KAPPA = 20.0


def _pts(n, seed):
    return W.sphere_points(n, seed=seed)


@pytest.mark.parametrize("k", [complex(1.0, 15.0), complex(0.0, -KAPPA)])
def test_gradient_kernel_is_odd(k):
    s = _pts(120, 0)
    t = _pts(90, 3) * 1.3
    for d in range(3):
        a = O.dense_matrix("grad_helmholtz", k, s, t, dx=d)
        b = O.dense_matrix("grad_helmholtz", k, t, s, dx=d)
        assert rel2(b.T, -a) <= 1e-14


def test_double_layer_is_normal_times_gradient():
    s = _pts(150, 0)
    t = _pts(110, 4) * 1.2
    n = s  # unit-sphere normals
    k = complex(1.0, 15.0)
    a = O.dense_matrix("double_layer", k, s, t, normals=n)
    g = sum(n[d][None, :] * O.dense_matrix("grad_helmholtz", k, s, t, dx=d) for d in range(3))
    assert rel2(g, a) <= 1e-13


def test_combined_field_decomposition():
    s = _pts(150, 0)
    t = _pts(110, 4) * 1.2
    n = s
    a = O.dense_matrix("combined_field", KAPPA, s, t, normals=n)
    g = sum(n[d][None, :] * O.dense_matrix("grad_helmholtz", complex(0, -KAPPA), s, t, dx=d)
            for d in range(3))
    h = O.dense_matrix("helmholtz", KAPPA, s, t)
    assert rel2(-g - 1j * KAPPA * h, a) <= 1e-13


def _oracle_adjoint(name, k, srcs, tgts, w, order, leaf):
    """The library's composition restated on oracle operators (roles exchanged)."""
    def op(kind, kk, dx=-1):
        o = O.OracleOperator(kind, kk, leaf, order)
        if dx >= 0:
            o.set_dx(dx)
        o.init(tgts, srcs)
        return o

    if name == "laplace":
        return op("laplace", 0.0).mult(w)
    if name in ("helmholtz", "modified_helmholtz"):
        return np.conj(op(name, k).mult(np.conj(w)))
    if name == "grad_helmholtz":
        return -np.conj(op(name, k, 0).mult(np.conj(w)))
    n = srcs
    if name == "double_layer":
        z = [op("grad_helmholtz", k, d).mult(np.conj(w)) for d in range(3)]
        return -np.conj(sum(n[d] * z[d] for d in range(3)))
    z = [op("grad_helmholtz", complex(0, -k.real), d).mult(np.conj(w)) for d in range(3)]
    y = op("helmholtz", k.real).mult(np.conj(w))
    return np.conj(sum(n[d] * z[d] for d in range(3)) - 1j * k.real * y)


def _gpu(name, order, leaf, srcs, tgts, dx=-1):
    g = make_gpu_op(name, leaf=leaf, order=order, dx=dx)
    if KERNELS[name][2]:
        g.init(srcs, tgts, srcs)
    else:
        g.init(srcs, tgts)
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(KERNELS))
def test_adjoint_parity_with_oracle_composition(name):
    ns, nt = 5000, 4000
    srcs = _pts(ns, 0)
    tgts = _pts(nt, 7) * 1.1
    dx = 0 if name == "grad_helmholtz" else -1
    g = _gpu(name, 8, 50, srcs, tgts, dx)
    w = densities_for(name, nt, seed=3)
    u = g.mult_adjoint(w)
    assert u.shape == (ns,)
    k = complex(KERNELS[name][1])
    uo = _oracle_adjoint(name, k, srcs, tgts, w, 8, 50)
    assert rel2(u, uo) <= 1e-12, rel2(u, uo)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(KERNELS))
@pytest.mark.parametrize("same_points", [True, False])
def test_adjoint_against_dense_matrix(name, same_points):
    ns = 1800
    srcs = _pts(ns, 0)
    tgts = srcs if same_points else _pts(1500, 9) * 1.15
    nt = tgts.shape[1]
    dx = 1 if name == "grad_helmholtz" else -1
    g = _gpu(name, 10, 40, srcs, tgts, dx)
    k = complex(KERNELS[name][1])
    a = O.dense_matrix(name, k, srcs, tgts, normals=srcs if KERNELS[name][2] else None, dx=dx)
    w = densities_for(name, nt, seed=4)
    u = g.mult_adjoint(w)
    ref = a.conj().T @ w
    if name == "laplace":
        ref = ref.real
    # as accurate as the forward matvec of the same operator
    v = densities_for(name, ns, seed=5)
    av = g.mult(v)
    e_fwd = rel2(av, a @ v if name != "laplace" else (a @ v).real)
    assert rel2(u, ref) <= max(2e-6, 5 * e_fwd), (rel2(u, ref), e_fwd)
    # <A v, w> = <v, A^H w> up to the IFGF error of both products
    lhs = np.vdot(w, av)
    rhs = np.vdot(u, v)
    assert abs(lhs - rhs) <= max(1e-5, 10 * e_fwd) * abs(lhs)


@pytest.mark.gpu
def test_adjoint_batch_and_mixed_precision():
    n = 6000
    pts = _pts(n, 0)
    g = _gpu("combined_field", 8, 50, pts, pts)
    w = np.stack([densities_for("combined_field", n, seed=s) for s in (1, 2)])
    u = g.mult_adjoint(w)
    assert rel2(u[1], g.mult_adjoint(w[1])) <= 1e-15
    g.set_precision("mixed")
    # the combined-field adjoint adds three mixed-precision gradient matvecs
    # and a Helmholtz one whose sum partly cancels (normal derivative against
    # i kappa times the single layer), so its relative error is several times
    # that of the forward kernel's fused mixed pipeline (1.3e-4 measured)
    assert rel2(g.mult_adjoint(w[0]), u[0]) <= 3e-4
