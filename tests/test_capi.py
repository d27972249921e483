"""The C ABI library loads, exports every symbol include/ifgf_b200.h
declares, and validates arguments on the host (no GPU work)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import ifgf_b200 as G
from ifgf_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "ifgf_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ifgf_[a-z_0-9]+)\s*\(", txt)) - {"ifgf_cutoff_fn"})


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(_lib.EXPORTED) == syms


def test_invalid_arguments_are_rejected():
    with pytest.raises(G.IfgfError) as e:
        G.HelmholtzIfgfOperator(1.0, 0, 8)
    assert e.value.code == 1
    with pytest.raises(G.IfgfError):
        G.HelmholtzIfgfOperator(1.0, 100, 0)
    with pytest.raises(G.IfgfError):
        G.HelmholtzIfgfOperator(float("nan"), 100, 8)
    op = G.GradHelmholtzIfgfOperator(1 + 2j, 100, 8)
    with pytest.raises(G.IfgfError):
        op.setDx(3)
    op.setDx(2)
    with pytest.raises(G.IfgfError) as e:
        op.set_precision(7)
    assert e.value.code == 1


def test_mult_before_init_is_a_state_error():
    op = G.LaplaceIfgfOperator(100, 8)
    with pytest.raises(ValueError):
        op.mult(np.zeros(3))  # size check on the host
    op._n_src = 3
    with pytest.raises(G.IfgfError) as e:
        op.mult(np.zeros(3))
    assert e.value.code == 3


def test_bad_points_rejected_before_gpu_work():
    op = G.LaplaceIfgfOperator(100, 8)
    p = np.zeros((3, 10))
    p[1, 4] = np.inf
    with pytest.raises(G.IfgfError) as e:
        op.init_plan_only(p, p)
    assert e.value.code == 1
    with pytest.raises(ValueError):
        op.init_plan_only(np.zeros((2, 10)), np.zeros((3, 10)))


def test_low_order_rejected_for_unclamped_kernels():
    # Laplace's low-order radial order is p-6 (laplace_ifgf.hpp:139-142):
    # p = 6 would give order 0, which the reference silently accepts
    p = np.random.default_rng(0).normal(size=(3, 50))
    op = G.LaplaceIfgfOperator(10, 6)
    with pytest.raises(G.IfgfError):
        op.init_plan_only(p, p)


def test_reference_names_present():
    from ifgf_b200 import pyifgf

    for name in ("MofifiedHelmholtzIfgfOperator", "GradHelmholtzIfgfOperator", "LaplaceIfgfOperator"):
        assert hasattr(pyifgf, name)
    assert G.MofifiedHelmholtzIfgfOperator is G.ModifiedHelmholtzIfgfOperator
    assert pyifgf.ModifiedHelmholtzIfgfOperator is pyifgf.MofifiedHelmholtzIfgfOperator
