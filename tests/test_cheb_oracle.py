"""Closed-form checks of the oracle's Chebyshev building blocks
(chebinterp.hpp:26-39 nodes, :176-250 chebtransform, :252-346 Clenshaw)."""
import numpy as np
import numpy.polynomial.chebyshev as npc

from oracle import oracle as O


def test_nodes_closed_form():
    for n in (1, 2, 5, 8, 13):
        x = O.cheb_nodes(n)
        ref = np.cos((2 * np.arange(n) + 1) / (2 * n) * np.pi)
        assert np.allclose(x, ref, rtol=0, atol=1e-15)


def _tensor_nodes(ns):
    r, t, p = (O.cheb_nodes(n) for n in ns)
    # index = iphi*nT*nR + jtheta*nR + kr  (chebinterp.hpp:101-112)
    P, T, R = np.meshgrid(p, t, r, indexing="ij")
    return np.stack([R.ravel(), T.ravel(), P.ravel()], axis=1)


def test_chebtransform_recovers_coefficients():
    rng = np.random.default_rng(0)
    ns = (3, 5, 4)
    c = rng.standard_normal(ns[::-1]) + 1j * rng.standard_normal(ns[::-1])  # [k][j][i]
    x = _tensor_nodes(ns)
    # values of sum c[k,j,i] T_i(x0) T_j(x1) T_k(x2) at the nodes
    vals = npc.chebval3d(x[:, 2], x[:, 1], x[:, 0], c.transpose(0, 1, 2))
    # chebval3d(x,y,z,c) uses c[i,j,k] T_i(x)T_j(y)T_k(z); we passed (z, y, x)
    coef = O.chebtransform3(np.array(ns), vals)
    assert np.allclose(coef, c.ravel(), atol=1e-13)


def test_clenshaw_matches_numpy_chebval():
    rng = np.random.default_rng(1)
    for ns in [(2, 5, 5), (5, 8, 8), (1, 2, 3), (4, 1, 2)]:
        c = rng.standard_normal(ns[::-1]) + 1j * rng.standard_normal(ns[::-1])
        x = rng.uniform(-1, 1, size=(50, 3))
        got = O.clenshaw3(np.array(ns), c.ravel(), x)
        ref = npc.chebval3d(x[:, 2], x[:, 1], x[:, 0], c)
        assert np.allclose(got, ref, atol=1e-12), ns


def test_transform_then_evaluate_interpolates():
    """test/test_chebinterp.cpp restated: interpolate exp(|x|^2 + z) on [-1,1]^3."""
    f = lambda p: np.exp(np.sum(p * p, axis=1) + p[:, 2])  # noqa: E731
    pts = np.random.default_rng(2).uniform(-1, 1, size=(1000, 3))
    rms = []
    for n in (8, 12, 16):
        ns = (n, n, n)
        coef = O.chebtransform3(np.array(ns), f(_tensor_nodes(ns)).astype(np.complex128))
        approx = O.clenshaw3(np.array(ns), coef, pts)
        rms.append(np.sqrt(np.mean(np.abs(approx - f(pts)) ** 2)))
    # spectral convergence of the interpolant of an entire function
    assert rms[2] < 1e-7 and rms[1] < rms[0] / 20 and rms[2] < rms[1] / 20, rms
