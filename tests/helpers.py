"""Shared helpers of the test-suite: kernel table and operator factories."""
import numpy as np

from ifgf_b200 import workloads as W

# name -> (product class name, wavenumber used in the tests, needs normals)
KERNELS = {
    "laplace": ("LaplaceIfgfOperator", 0.0, False),
    "helmholtz": ("HelmholtzIfgfOperator", 20.0, False),
    "modified_helmholtz": ("ModifiedHelmholtzIfgfOperator", complex(2.35318922187804, 43.6495537831048), False),
    "grad_helmholtz": ("GradHelmholtzIfgfOperator", complex(1.0, 15.0), False),
    "double_layer": ("DoubleLayerHelmholtzIfgfOperator", complex(1.0, 15.0), True),
    "combined_field": ("CombinedFieldHelmholtzIfgfOperator", 20.0, True),
}


def make_gpu_op(name, leaf=64, order=8, dx=-1, k=None):
    import ifgf_b200 as G

    cls_name, k0, _ = KERNELS[name]
    k = k0 if k is None else k
    cls = getattr(G, cls_name)
    if name == "laplace":
        op = cls(leaf, order)
    else:
        op = cls(k, leaf, order)
    if name == "grad_helmholtz":
        op.setDx(dx)
    return op


def make_oracle_op(name, leaf=64, order=8, dx=-1, k=None):
    from oracle import oracle as O

    k = KERNELS[name][1] if k is None else k
    op = O.OracleOperator(name, k, leaf, order)
    if name == "grad_helmholtz":
        op.set_dx(dx)
    return op


def init_op(op, name, srcs, tgts):
    if KERNELS[name][2]:
        op.init(srcs, tgts, srcs)  # unit-sphere normals = the points themselves
    else:
        op.init(srcs, tgts)


def rel2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def densities_for(name, n, seed=1):
    return W.densities(n, complex_=(name != "laplace"), seed=seed)
