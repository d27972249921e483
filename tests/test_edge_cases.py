"""Degenerate inputs through the whole pipeline.

The FP64 matvec must match the oracle (relative 2-norm <= 1e-12, or to
1e-14 absolute where the result is zero) on point sets that reach the
corners of the tree build, the interaction lists and the far field: single
points, fewer points than a leaf, exact duplicates (self pairs contribute
zero), a flat set, clusters so far apart that everything between them is far
field, and targets that lie on no source box.  The mixed pipeline follows
FP64 within its tolerance and a batch of two equals two single matvecs.
A lone source is a one-box tree of side ~1e-8 (the inflated bounding box of
one point), so a distant target has s = H / r below the interpolation
domain's lower bound 1e-4 and contributes zero -- the reference's rule for
points outside every cone (cone_domain.hpp:237-240), which both sides follow.
"""
import numpy as np
import pytest

from ifgf_b200 import workloads as W

from .helpers import densities_for, make_gpu_op, make_oracle_op, rel2

PARITY_TOL = 1e-12
MIXED_TOL = 5e-5


def _cases():
    rng = np.random.default_rng(11)
    dup = W.sphere_points(6000, seed=0)
    dup[:, 3000:4000] = dup[:, :1000]  # exact duplicates: zero self pairs
    flat = rng.standard_normal((3, 5000))
    flat[2] = 0.0
    ball = 0.05 * rng.standard_normal((3, 3000)) + np.array([[3.0], [0.0], [0.0]])
    shell = W.sphere_points(3000, seed=4)
    far_t = W.sphere_points(2000, seed=5) * 0.1 + np.array([[-4.0], [1.0], [0.5]])
    return [
        ("one_point", rng.standard_normal((3, 1)), rng.standard_normal((3, 1)) + 2.0),
        ("below_leaf", W.sphere_points(40, seed=1), W.sphere_points(40, seed=1)),
        ("duplicates", dup, dup),
        ("flat", flat, flat),
        ("separated_clusters", np.concatenate([ball, shell], axis=1),
         np.concatenate([ball, shell], axis=1)),
        ("targets_off_the_sources", shell, far_t),
    ]


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
@pytest.mark.parametrize("name", ["helmholtz", "laplace", "combined_field"])
def test_degenerate_point_sets(case, name):
    _, src, tgt = case
    n = src.shape[1]
    w = densities_for(name, n)
    g = make_gpu_op(name, leaf=64, order=8)
    o = make_oracle_op(name, leaf=64, order=8)
    if name == "combined_field":
        nrm = src / np.maximum(np.linalg.norm(src, axis=0), 1e-300)
        g.init(src, tgt, nrm)
        o.init(src, tgt, nrm)
    else:
        g.init(src, tgt)
        o.init(src, tgt)
    ug, uo = g.mult(w), o.mult(w)
    scale = max(np.linalg.norm(uo), 1e-300)
    assert np.linalg.norm(ug - uo) <= PARITY_TOL * scale + 1e-14, (name, case[0])
    assert g.stats()["missing_cone_lookups"] == 0
    if np.linalg.norm(uo) > 0:
        g.set_precision("mixed")
        assert rel2(g.mult(w), ug) <= MIXED_TOL, (name, case[0])
        w2 = np.stack([w, densities_for(name, n, seed=9)])
        ub = g.mult_batch(w2)
        assert rel2(ub[0], g.mult(w2[0])) <= 1e-6
        assert rel2(ub[1], g.mult(w2[1])) <= 1e-6
