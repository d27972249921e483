"""Generates tests/golden/*.npz: seeded small IFGF cases for every kernel.

Each file holds the inputs' parameters, the oracle's matvec at 100 sampled
targets and the FP64 direct sum at the same targets.  The reference cannot be
built in this image (Eigen >= 5 and oneTBB are absent), so these fixtures pin
the oracle restatement against regressions and give the CUDA path fixed
vectors to match; the direct-sum values are independent of IFGF.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ifgf_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    "laplace": (0.0, -1),
    "helmholtz": (20.0, -1),
    "modified_helmholtz": (complex(2.35318922187804, 43.6495537831048), -1),
    "grad_helmholtz": (complex(1.0, 15.0), 1),
    "double_layer": (complex(1.0, 15.0), -1),
    "combined_field": (20.0, -1),
}
N, LEAF, ORDER, NT = 2000, 40, 8, 100


def make(name):
    k, dx = CASES[name]
    pts = W.sphere_points(N, seed=0)
    w = W.densities(N, complex_=(name != "laplace"), seed=1)
    idx = W.sample_targets(N, NT, seed=2)
    normals = pts if name in ("double_layer", "combined_field") else None
    op = O.OracleOperator(name, k, LEAF, ORDER)
    if dx != -1:
        op.set_dx(dx)
    op.init(pts, pts, normals)
    u = op.mult(w)[idx]
    d = O.direct_sum(name, k, pts, w, pts, idx, normals=normals, dx=dx)
    np.savez(os.path.join(HERE, f"{name}.npz"), n=N, leaf=LEAF, order=ORDER, k=complex(k), dx=dx,
             idx=idx, u=u, direct=d)


if __name__ == "__main__":
    for name in CASES:
        make(name)
        print("wrote", name)
