"""The tensor-core upward transfer (tcgen05 split-TF32 kernel) against the
FP32-FMA upward kernels and the FP64 oracle, through the C ABI.

Both mixed pipelines compute the same interpolants in FP32 arithmetic; the
tensor-core form sums the tensor-product basis in another order and with
the TF32 split ((A_hi + A_lo)(B_hi + B_lo)), so the two agree to FP32
rounding, and both stay within the mixed tolerance of the FP64 pipeline
(the transfer is transferInterp, ifgfoperator.hpp:1639-1705).
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W

from .helpers import KERNELS, densities_for, init_op, make_gpu_op, make_oracle_op, rel2

TC_VS_FFMA = 2e-6  # tensor-core vs FFMA upward, same mixed pipeline otherwise
MIXED_TOL = 2e-5   # mixed pipeline vs the FP64 oracle


def _three_paths(g, w, batch=None):
    out = {}
    for path in ("ffma", "tensor", "auto"):
        g.set_upward_path(path)
        out[path] = g.mult_batch(w) if batch else g.mult(w)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("order", [8, 9])
def test_tensor_upward_matches_ffma_and_oracle(order):
    n = 30000
    pts = W.ellipsoid_points(n, seed=0)
    w = W.densities(n, seed=1)
    g = make_gpu_op("helmholtz", leaf=60, order=order, k=60.0)
    o = make_oracle_op("helmholtz", leaf=60, order=order, k=60.0)
    g.init(pts, pts)
    o.init(pts, pts)
    uo = o.mult(w)
    g.set_precision("mixed")
    u = _three_paths(g, w)
    assert rel2(u["tensor"], u["ffma"]) <= TC_VS_FFMA, rel2(u["tensor"], u["ffma"])
    assert rel2(u["auto"], u["ffma"]) <= TC_VS_FFMA
    # as close to the FP64 oracle as the FFMA mixed pipeline (whose FP32
    # error at this wavenumber and order is its own, ~5e-4 at p = 8)
    e_ffma = rel2(u["ffma"], uo)
    for path in u:
        assert rel2(u[path], uo) <= 1.02 * e_ffma + 1e-6, (path, rel2(u[path], uo), e_ffma)
    assert g.stats()["missing_cone_lookups"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(KERNELS))
def test_tensor_upward_all_kernels(name):
    """Every plug-in's centre-shift factor through the tensor-core kernel
    (forced on every level): same result as the FFMA kernel."""
    n = 8000
    pts = W.sphere_points(n, seed=0)
    w = densities_for(name, n)
    dxs = [-1, 1] if name == "grad_helmholtz" else [-1]
    for dx in dxs:
        g = make_gpu_op(name, leaf=40, order=8, dx=dx)
        init_op(g, name, pts, pts)
        u64 = g.mult(w)
        g.set_precision("mixed")
        u = _three_paths(g, w)
        assert rel2(u["tensor"], u["ffma"]) <= TC_VS_FFMA, (name, dx, rel2(u["tensor"], u["ffma"]))
        assert rel2(u["tensor"], u64) <= MIXED_TOL, (name, dx, rel2(u["tensor"], u64))


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [4, 8, 13])
def test_tensor_upward_batched(batch):
    """Batched right-hand sides: rows of a tile are (cone, plane) pairs."""
    n = 20000
    pts = W.ellipsoid_points(n, seed=0)
    g = make_gpu_op("helmholtz", leaf=60, order=9, k=50.0)
    g.init(pts, pts)
    g.set_precision("mixed")
    wb = np.stack([W.densities(n, seed=10 + b) for b in range(batch)])
    u = _three_paths(g, wb, batch=True)
    assert rel2(u["tensor"], u["ffma"]) <= TC_VS_FFMA, rel2(u["tensor"], u["ffma"])
    # plane b equals the single right-hand-side matvec of density b
    g.set_upward_path("tensor")
    for b in (0, batch - 1):
        assert rel2(u["tensor"][b], g.mult(wb[b])) <= TC_VS_FFMA


@pytest.mark.gpu
def test_tensor_upward_repeatable():
    n = 20000
    pts = W.ellipsoid_points(n, seed=0)
    g = make_gpu_op("helmholtz", leaf=60, order=9, k=50.0)
    g.init(pts, pts)
    g.set_precision("mixed")
    g.set_upward_path("tensor")
    w = W.densities(n, seed=1)
    a = g.mult(w)
    assert np.array_equal(a, g.mult(w))  # no atomics: the same bits every call


@pytest.mark.gpu
def test_bounded_wait_gives_up_with_timeout_status():
    """The bounded wait of the tensor-core kernels: a barrier nothing arrives
    at makes the wait give up after its limit with IFGF_ERR_TIMEOUT, and the
    device stays usable."""
    import ctypes as C

    from ifgf_b200 import _lib

    waited = C.c_double(0)
    rc = _lib.lib.ifgf_bounded_wait_selftest(50.0, C.byref(waited))
    assert rc == 5, _lib.lib.ifgf_last_error()
    assert 50.0 <= waited.value < 5000.0
    # a matvec after it still works
    n = 3000
    pts = W.sphere_points(n, seed=0)
    g = make_gpu_op("laplace", leaf=50, order=8)
    g.init(pts, pts)
    o = make_oracle_op("laplace", leaf=50, order=8)
    o.init(pts, pts)
    w = W.densities(n, complex_=False, seed=1)
    assert rel2(g.mult(w), o.mult(w)) <= 1e-12


@pytest.mark.gpu
def test_autotuner_records_a_choice_per_level_and_plane_count():
    """The AUTO path times both upward kernels once per plane count on the
    operator's own tables and keeps the faster per level; the choice and the
    times are reported in the stats, and results match the FFMA path."""
    n = 30000
    pts = W.ellipsoid_points(n, seed=0)
    g = make_gpu_op("helmholtz", leaf=60, order=9, k=60.0)
    g.init(pts, pts)
    g.set_precision("mixed")
    w = W.densities(n, seed=1)
    wb = np.stack([W.densities(n, seed=20 + b) for b in range(8)])
    u1, ub = g.mult(w), g.mult_batch(wb)
    tuner = g.stats()["upward_tuner"]
    assert "1" in tuner and "8" in tuner, tuner.keys()
    for planes, rec in tuner.items():
        timed = [i for i, c in enumerate(rec["tensor"]) if c >= 0]
        assert timed, planes
        for i in timed:
            assert rec["ms_ffma"][i] > 0 and rec["ms_tensor"][i] > 0
            assert rec["tensor"][i] == (1 if rec["ms_tensor"][i] < 0.97 * rec["ms_ffma"][i] else 0)
    g.set_upward_path("ffma")
    assert rel2(u1, g.mult(w)) <= TC_VS_FFMA
    assert rel2(ub, g.mult_batch(wb)) <= TC_VS_FFMA


@pytest.mark.gpu
def test_tensor_upward_basis_images_follow_the_wavenumber():
    """The basis images of the tensor-core kernel (built once per level)
    carry the centre-shift factors of the operator's wavenumber: after
    set_wavenumber on the same cone grids the matvec equals a fresh
    operator's at the new wavenumber."""
    import ifgf_b200 as G

    n = 60000
    pts = W.sphere_points(n, seed=0)
    w = W.densities(n, seed=1)
    k1, k2 = 20.2, 20.6  # the same cone grids on every level
    g = G.HelmholtzIfgfOperator(k1, 60, 9)
    g.init(pts, pts)
    g.set_precision("mixed")
    g.set_upward_path("tensor")
    g.mult(w)
    assert sum(g.stats()["upward_images_bytes"]) > 0
    g.set_wavenumber(k2)
    assert g.stats()["far_plan"]["built"] in (0, 1)
    u = g.mult(w)
    f = G.HelmholtzIfgfOperator(k2, 60, 9)
    f.init(pts, pts)
    f.set_precision("mixed")
    f.set_upward_path("tensor")
    assert rel2(u, f.mult(w)) <= 1e-14, rel2(u, f.mult(w))
