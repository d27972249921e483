"""Seeded synthetic point sets and densities for the IFGF matvec.

Points are normalised i.i.d. standard-normal 3-vectors (uniform on the unit
sphere); the ellipsoid variant projects them radially onto the surface with
semi-axes ``axes``.  Arrays are float64 with shape (3, N), the layout of the
reference's ``Eigen::Array<double, 3, Dynamic>`` point arrays.
"""
import numpy as np


def sphere_points(n, seed=0):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return np.ascontiguousarray(v.T)


def ellipsoid_points(n, axes=(1.0, 1.0, 0.5), seed=0):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    a = np.asarray(axes, dtype=np.float64)
    scale = 1.0 / np.sqrt(np.sum(v * v / (a * a), axis=1))
    return np.ascontiguousarray((v * scale[:, None]).T)


def densities(n, complex_=True, seed=1, batch=None):
    rng = np.random.default_rng(seed)
    shape = (n,) if batch is None else (batch, n)
    if complex_:
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return rng.standard_normal(shape)


def sample_targets(m, k=1000, seed=2):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(m, size=min(k, m), replace=False))
