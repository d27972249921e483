"""Committed fixtures (tests/golden/make_golden.py): the oracle reproduces
them (regression pin) and the CUDA path matches them to 1e-12; the fixtures'
direct sums bound the IFGF error."""
import os

import numpy as np
import pytest

from ifgf_b200 import workloads as W
from oracle import oracle as O

from .helpers import KERNELS, make_gpu_op, rel2

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = list(KERNELS)


def _load(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    return {k: z[k] for k in z.files}


def _inputs(name, g):
    n = int(g["n"])
    pts = W.sphere_points(n, seed=0)
    w = W.densities(n, complex_=(name != "laplace"), seed=1)
    return pts, w


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name):
    g = _load(name)
    pts, w = _inputs(name, g)
    k, dx = complex(g["k"]), int(g["dx"])
    op = O.OracleOperator(name, k, int(g["leaf"]), int(g["order"]))
    if dx != -1:
        op.set_dx(dx)
    normals = pts if KERNELS[name][2] else None
    op.init(pts, pts, normals)
    u = op.mult(w)[g["idx"]]
    assert rel2(u, g["u"]) < 1e-13
    d = O.direct_sum(name, k, pts, w, pts, g["idx"], normals=normals, dx=dx)
    assert rel2(d, g["direct"]) < 1e-14
    assert rel2(g["u"], g["direct"]) < 2e-2


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_golden(name):
    g = _load(name)
    pts, w = _inputs(name, g)
    dx = int(g["dx"])
    op = make_gpu_op(name, leaf=int(g["leaf"]), order=int(g["order"]), dx=dx, k=complex(g["k"])
                     if name not in ("laplace", "helmholtz", "combined_field") else float(np.real(g["k"])))
    if KERNELS[name][2]:
        op.init(pts, pts, pts)
    else:
        op.init(pts, pts)
    u = op.mult(w)[g["idx"]]
    assert rel2(u, g["u"]) <= 1e-12
    d = op.direct_eval(w, g["idx"])
    assert rel2(d, g["direct"]) < 1e-13
