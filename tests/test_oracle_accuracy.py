"""The oracle against the FP64 dense direct sum (the reference's own accuracy
study, test/test_ifgf.cpp:143-165, restated with asserted bounds)."""
import numpy as np
import pytest

from ifgf_b200 import workloads as W
from oracle import oracle as O

from .helpers import KERNELS, densities_for, make_oracle_op, rel2

# error bounds at N = 4000, leaf 50, order 8 (measured ~1e-4 .. 3e-3)
BOUNDS = {
    "laplace": 2e-3,
    "helmholtz": 2e-3,
    "modified_helmholtz": 2e-2,
    "grad_helmholtz": 2e-2,
    "double_layer": 2e-2,
    "combined_field": 2e-2,
}


@pytest.mark.parametrize("name", list(KERNELS))
def test_oracle_vs_direct(name):
    n = 4000
    pts = W.sphere_points(n, seed=0)
    w = densities_for(name, n)
    op = make_oracle_op(name, leaf=50, order=8)
    normals = pts if KERNELS[name][2] else None
    op.init(pts, pts, normals)
    u = op.mult(w)
    idx = W.sample_targets(n, 200, seed=2)
    d = O.direct_sum(name, KERNELS[name][1], pts, w, pts, idx, normals=normals)
    assert rel2(u[idx], d) < BOUNDS[name], rel2(u[idx], d)


def test_oracle_converges_in_order():
    n = 6000
    pts = W.sphere_points(n, seed=0)
    w = W.densities(n, complex_=False, seed=1)
    idx = W.sample_targets(n, 200, seed=2)
    d = O.direct_sum("laplace", 0, pts, w, pts, idx)
    errs = []
    for p in (8, 10):
        op = O.OracleOperator("laplace", 0, 50, p)
        op.init(pts, pts)
        errs.append(rel2(op.mult(w)[idx], d))
    assert errs[1] < errs[0] / 20, errs


def test_oracle_connectivity():
    """Every (source, target) pair is covered exactly once by the near and
    far lists (the reference's CHECK_CONNECTIVITY, ifgfoperator.hpp:285-290)."""
    n = 3000
    src = W.sphere_points(n, seed=0)
    tgt = W.ellipsoid_points(1500, axes=(1.2, 1.1, 0.8), seed=4)
    op = O.OracleOperator("laplace", 0, 40, 8)
    op.init(src, tgt)
    cov = np.zeros((n, 1500), dtype=np.int32)
    for lvl in range(op.levels()):
        ints, _ = op.boxes(lvl)
        for b in range(len(ints)):
            s0, s1 = ints[b, 0], ints[b, 1]
            for far in (0, 1):
                for t0, t1 in op.interaction_list(lvl, b, far):
                    cov[s0:s1, t0:t1] += 1
    assert cov.min() == 1 and cov.max() == 1
