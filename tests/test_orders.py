"""Tolerance-driven interpolation orders (tol > 0).

IfgfOperator::init with tol > 0 (ifgfoperator.hpp:80-85) replaces the fixed
orders by estimateRefinement (ifgfoperator.hpp:108-244): on ten boxes of the
deepest source level, the order of each dimension grows while Chebyshev layer
n - 3 of the order + 4 expansion of the box's factored kernel on coarse cone 0
holds more than tol of the coefficient norm.

CPU: the oracle's C++ estimate against an independent numpy restatement of
the same steps (Laplace, Helmholtz), the loose-tolerance and monotonicity
properties, and the plan-only refusal.  GPU: the product's estimate (kernel
values from the GPU probe) equals the oracle's for every kernel, and the
matvec on the estimated orders keeps FP64 parity with the oracle.
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W

from .helpers import KERNELS, densities_for, init_op, rel2


def _oracle(name, k=None, leaf=64, order=5, tol=-1.0):
    from oracle import oracle as O

    k = KERNELS[name][1] if k is None else k
    return O.OracleOperator(name, k, leaf, order, tol=tol)


def _gpu(name, k=None, leaf=64, order=5, tol=-1.0):
    import ifgf_b200 as G

    cls_name, k0, _ = KERNELS[name]
    k = k0 if k is None else k
    cls = getattr(G, cls_name)
    if name == "laplace":
        return cls(leaf, order, 1, tol)
    return cls(k, leaf, order, 1, tol)


def _cheb_matrix(n):
    j = np.arange(n)
    T = np.cos(np.outer(j, np.pi * (2 * j + 1) / (2 * n)))  # T[k, j] = T_k(x_j)
    T *= np.where(j == 0, 1.0, 2.0)[:, None] / n
    return T


def _numpy_estimate(name, k, pts_sorted, ints, bb, p, tol):
    """The estimate restated with numpy for the Laplace and Helmholtz kernels."""
    nb = len(ints)
    stride = nb // 10
    best = np.zeros(3, dtype=int)
    for i in range(10):
        b = i * stride
        f, l = ints[b, 0], ints[b, 1]
        mn, mx = bb[b, :3], bb[b, 3:]
        xc = (mn + mx) / 2
        H = np.max(np.abs(mx - mn))
        src = pts_sorted[f:l]
        base = np.zeros(3, dtype=int)
        err = np.full(3, np.inf)
        newp = p + base
        while err.max() > tol and base.max() < 10:
            newp = p + base
            n = newp + 4
            if name == "laplace":
                ne = np.array([1, 2, 4])
            else:
                ne = np.array([1, 2, 4]) * int(np.ceil(max(k * H / 4.0, 1.0)))
            lo = np.array([1e-4, 0.0, -np.pi])
            hi = np.array([np.sqrt(3.0) / 3, np.pi, np.pi])
            h = (hi - lo) / ne
            x = [np.cos((2 * np.arange(n[d]) + 1) / (2.0 * n[d]) * np.pi) * h[d] / 2 + lo[d] + h[d] / 2
                 for d in range(3)]
            s2, s1, s0 = np.meshgrid(x[2], x[1], x[0], indexing="ij")  # r fastest
            r = H / s0
            y = np.stack([xc[0] + r * np.cos(s2) * np.sin(s1), xc[1] + r * np.sin(s2) * np.sin(s1),
                          xc[2] + r * np.cos(s1)], axis=-1).reshape(-1, 3)
            dc = np.linalg.norm(y - xc, axis=1)
            d = np.linalg.norm(src[None, :, :] - y[:, None, :], axis=2)
            if name == "laplace":
                v = (dc[:, None] / d).sum(axis=1).astype(complex)
            else:
                v = (np.exp(1j * k * (d - dc[:, None])) * dc[:, None] / d).sum(axis=1)
            c = v.reshape(n[2], n[1], n[0])
            c = np.einsum("kj,abj->abk", _cheb_matrix(n[0]), c)
            c = np.einsum("kj,ajb->akb", _cheb_matrix(n[1]), c)
            c = np.einsum("kj,jab->kab", _cheb_matrix(n[2]), c)
            m2 = np.abs(c) ** 2
            tot = max(1.0, np.sqrt(m2.sum()))
            err = np.array([np.sqrt(m2[:, :, n[0] - 3].sum()), np.sqrt(m2[:, n[1] - 3, :].sum()),
                            np.sqrt(m2[n[2] - 3, :, :].sum())]) / tot
            base = base + (err > tol)
        best = np.maximum(best, newp)
    return best


@pytest.mark.parametrize("name,k", [("laplace", 0.0), ("helmholtz", 16.0)])
@pytest.mark.parametrize("tol", [1e-4, 1e-6])
def test_oracle_estimate_matches_numpy_restatement(name, k, tol):
    n, p = 8000, 5
    pts = W.sphere_points(n, seed=0)
    o = _oracle(name, k=k, leaf=64, order=p, tol=tol)
    o.init(pts, pts)
    lvl = o.levels() - 1
    ints, bb = o.boxes(lvl)
    pts_sorted = pts.T[o.perm()]
    ref = _numpy_estimate(name, k, pts_sorted, ints, bb, p, tol)
    assert o.orders(1).tolist() == ref.tolist()
    assert o.orders(0).tolist() == (ref - 3).tolist()


@pytest.mark.parametrize("name", list(KERNELS))
def test_loose_tolerance_keeps_the_constructor_order(name):
    # every layer test passes at once: orders (p, p, p), with no radial
    # reduction (the fixed-order path would give (p - 3, p, p))
    pts = W.sphere_points(5000, seed=0)
    o = _oracle(name, leaf=64, order=8, tol=0.5)
    init_op(o, name, pts, pts)
    assert o.orders(1).tolist() == [8, 8, 8]
    f = _oracle(name, leaf=64, order=8)
    init_op(f, name, pts, pts)
    assert f.orders(1).tolist() == [5, 8, 8]


@pytest.mark.parametrize("name", ["helmholtz", "combined_field"])
def test_orders_grow_as_the_tolerance_shrinks(name):
    pts = W.sphere_points(8000, seed=0)
    prev = None
    for tol in (1e-2, 1e-4, 1e-6, 1e-8):
        o = _oracle(name, leaf=64, order=5, tol=tol)
        init_op(o, name, pts, pts)
        cur = o.orders(1)
        if prev is not None:
            assert np.all(cur >= prev), (tol, cur, prev)
        prev = cur
    assert prev.sum() > 15  # 1e-8 needs more than the starting (5, 5, 5)


def test_oracle_error_follows_the_tolerance():
    n = 8000
    pts = W.sphere_points(n, seed=0)
    w = densities_for("helmholtz", n)
    idx = W.sample_targets(n, 300, seed=2)
    from oracle import oracle as O

    d = O.direct_sum("helmholtz", 16.0, pts, w, pts, idx)
    errs = []
    for tol in (1e-3, 1e-6):
        o = _oracle("helmholtz", k=16.0, leaf=64, order=5, tol=tol)
        o.init(pts, pts)
        errs.append(rel2(o.mult(w)[idx], d))
    # the estimate samples one cone with unit weights: a heuristic, not a
    # bound (measured 1.05e-3 and 1.15e-5 here)
    assert errs[1] < 0.05 * errs[0], errs
    assert errs[1] < 1e-4, errs


def test_plan_only_init_refuses_order_estimation():
    import ifgf_b200 as G

    pts = W.sphere_points(2000, seed=0)
    op = G.HelmholtzIfgfOperator(10.0, 64, 5, 1, 1e-6)
    with pytest.raises(Exception, match="tol > 0"):
        op.init_plan_only(pts, pts)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(KERNELS))
def test_gpu_estimated_orders_and_matvec_match_oracle(name):
    n = 6000
    pts = W.sphere_points(n, seed=0)
    w = densities_for(name, n)
    for tol in (1e-4, 1e-7):
        g = _gpu(name, leaf=50, order=5, tol=tol)
        o = _oracle(name, leaf=50, order=5, tol=tol)
        init_op(g, name, pts, pts)
        init_op(o, name, pts, pts)
        for step in (0, 1):
            assert g.orders(step).tolist() == o.orders(step).tolist(), (name, tol, step)
    # the last (finest) orders: FP64 parity with the oracle, mixed within its bound
    uo = o.mult(w)
    ug = g.mult(w)
    assert rel2(ug, uo) <= 1e-12, (name, rel2(ug, uo))
    g.set_precision("mixed")
    um = g.mult(w)
    assert rel2(um, ug) <= 5e-5, name
    # estimated orders are generally no batched shape: batches run the
    # single right-hand-side path and equal it
    ub = g.mult_batch(np.stack([w, densities_for(name, n, seed=7)]))
    assert rel2(ub[0], um) <= 1e-6, name
    assert g.stats()["missing_cone_lookups"] == 0


@pytest.mark.gpu
def test_set_wavenumber_re_estimates_the_orders():
    n = 8000
    pts = W.sphere_points(n, seed=0)
    w = densities_for("helmholtz", n)
    op = _gpu("helmholtz", k=5.0, leaf=64, order=5, tol=1e-6)
    op.init(pts, pts)
    for k in (5.5, 30.0):
        op.set_wavenumber(k)
        fresh = _gpu("helmholtz", k=k, leaf=64, order=5, tol=1e-6)
        fresh.init(pts, pts)
        assert op.orders(1).tolist() == fresh.orders(1).tolist(), k
        assert rel2(op.mult(w), fresh.mult(w)) <= 1e-14, k
