"""ctypes view of the CPU oracle (TEST INFRASTRUCTURE ONLY).

PARITY UNPINNED: the reference (TimHRO/ifgf) needs Eigen >= 5.0.1 and oneTBB,
which this image lacks, and its tests store no golden vectors; the oracle is
anchored by the FP64 direct sum, closed-form Chebyshev identities and the
connectivity check instead.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module.  Point arrays are float64 (3, N) as in the reference's Eigen API.
"""
import ctypes as C
import os

import numpy as np

from .build import LIB, build_oracle

_lib = None

KINDS = {
    "laplace": 0,
    "helmholtz": 1,
    "modified_helmholtz": 2,
    "grad_helmholtz": 3,
    "double_layer": 4,
    "combined_field": 5,
    # k-derivatives of kinds 1 and 5 (not reference kernels; see the C++ header)
    "helmholtz_dk": 6,
    "combined_field_dk": 7,
}

_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_long)
_ip = C.POINTER(C.c_int)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build_oracle()
        L = C.CDLL(LIB)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.c_int, C.c_double, C.c_double, C.c_long, C.c_int, C.c_long,
                                    C.c_double]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_set_dx.argtypes = [C.c_void_p, C.c_int]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_init.argtypes = [C.c_void_p, _dp, C.c_long, _dp, C.c_long, _dp]
        L.oracle_mult.argtypes = [C.c_void_p, _dp, _dp]
        L.oracle_mult_sample.argtypes = [C.c_void_p, _dp, C.c_int, _lp, C.c_long, _dp]
        L.oracle_mult_sample.restype = C.c_double
        L.oracle_work.argtypes = [C.c_void_p, C.c_int, _lp, C.c_long, _dp]
        L.oracle_max_threads.restype = C.c_int
        L.oracle_levels.argtypes = [C.c_void_p, C.c_int]
        L.oracle_num_boxes.restype = C.c_long
        L.oracle_num_boxes.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.oracle_rec_level.argtypes = [C.c_void_p]
        L.oracle_perm.argtypes = [C.c_void_p, C.c_int, _lp]
        L.oracle_boxes.argtypes = [C.c_void_p, C.c_int, C.c_int, _lp, _dp]
        L.oracle_list.restype = C.c_long
        L.oracle_list.argtypes = [C.c_void_p, C.c_int, C.c_long, C.c_int, _lp, C.c_long]
        L.oracle_cones.restype = C.c_long
        L.oracle_cones.argtypes = [C.c_void_p, C.c_int, C.c_long, C.c_int, _lp, C.c_long]
        L.oracle_grid.argtypes = [C.c_void_p, C.c_int, C.c_int, _lp]
        L.oracle_orders.argtypes = [C.c_void_p, C.c_int, _ip]
        L.oracle_direct.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, _dp, C.c_long, _dp,
                                    _dp, _dp, _lp, C.c_long, _dp]
        L.oracle_dense.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, _dp, C.c_long, _dp,
                                   _dp, C.c_long, _dp]
        L.oracle_cheb_nodes.argtypes = [C.c_int, _dp]
        L.oracle_chebtransform3.argtypes = [_ip, _dp, _dp]
        L.oracle_clenshaw3.argtypes = [_ip, _dp, _dp, C.c_long, _dp]
        L.oracle_morton_less.argtypes = [_dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def _aos(pts):
    """(3, N) -> contiguous AoS xyz (Eigen 3xN column-major memory)."""
    a = np.asarray(pts, dtype=np.float64)
    assert a.ndim == 2 and a.shape[0] == 3
    return np.ascontiguousarray(a.T)


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def set_threads(n):
    lib().oracle_set_threads(int(n))


def max_threads():
    return lib().oracle_max_threads()


class OracleOperator:
    """CPU restatement of IfgfOperator<...> (ifgfoperator.hpp) for one kernel."""

    def __init__(self, kind, k=0.0, leaf_size=100, order=8, n_elem=1, tol=-1.0):
        self.kind = KINDS[kind] if isinstance(kind, str) else int(kind)
        k = complex(k)
        self.k = k
        self.h = lib().oracle_create(self.kind, k.real, k.imag, leaf_size, order, n_elem, tol)
        self.n_src = self.n_tgt = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def set_dx(self, dx):
        lib().oracle_set_dx(self.h, int(dx))

    def init(self, srcs, tgts, normals=None):
        s = _aos(srcs)
        t = _aos(tgts)
        n = _aos(normals) if normals is not None else None
        self._keep = (s, t, n)
        lib().oracle_init(self.h, _p(s), s.shape[0], _p(t), t.shape[0],
                          _p(n) if n is not None else None)
        self.n_src, self.n_tgt = s.shape[0], t.shape[0]

    def mult(self, w):
        w = np.ascontiguousarray(np.asarray(w, dtype=np.complex128))
        out = np.zeros(self.n_tgt, dtype=np.complex128)
        lib().oracle_mult(self.h, _p(w.view(np.float64)), _p(out.view(np.float64)))
        return out.real.copy() if self.kind == 0 else out

    def mult_sample(self, w, level, boxes):
        """recursive_mult over the subtrees of the given source boxes of
        `level` (>= the recursive level) only: a bounded sample of the
        matvec, one subtree per thread; the result is partial."""
        w = np.ascontiguousarray(np.asarray(w, dtype=np.complex128))
        b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int64))
        out = np.zeros(self.n_tgt, dtype=np.complex128)
        busy = lib().oracle_mult_sample(self.h, _p(w.view(np.float64)), int(level), _p(b, _lp),
                                        len(b), _p(out.view(np.float64)))
        if busy < 0:
            raise ValueError("sample level must be >= the recursive level")
        self.last_busy_s = busy  # summed single-thread seconds of the sampled subtrees
        return out

    def work(self, level=None, boxes=None):
        """Modelled work [near pairs, leaf evals, far evals, upward evals] of
        the subtrees of the given boxes of `level` (None: the whole tree)."""
        out = np.zeros(4)
        if boxes is None:
            lib().oracle_work(self.h, 0, None, -1, _p(out))
        else:
            b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int64))
            lib().oracle_work(self.h, int(level), _p(b, _lp), len(b), _p(out))
        return out

    # ---- table dumps -------------------------------------------------
    def levels(self, which=0):
        return lib().oracle_levels(self.h, which)

    def num_boxes(self, level, which=0):
        return lib().oracle_num_boxes(self.h, which, level)

    def rec_level(self):
        return lib().oracle_rec_level(self.h)

    def perm(self, which=0):
        n = self.n_src if which == 0 else self.n_tgt
        out = np.zeros(n, dtype=np.int64)
        lib().oracle_perm(self.h, which, _p(out, _lp))
        return out

    def boxes(self, level, which=0):
        nb = self.num_boxes(level, which)
        ints = np.zeros((nb, 12), dtype=np.int64)
        bb = np.zeros((nb, 6), dtype=np.float64)
        lib().oracle_boxes(self.h, which, level, _p(ints, _lp), _p(bb))
        return ints, bb

    def interaction_list(self, level, box, far):
        n = lib().oracle_list(self.h, level, box, int(far), None, 0)
        out = np.zeros((max(n, 1), 2), dtype=np.int64)
        lib().oracle_list(self.h, level, box, int(far), _p(out, _lp), n)
        return out[:n]

    def cones(self, level, box, step):
        n = lib().oracle_cones(self.h, level, box, step, None, 0)
        out = np.zeros(max(n, 1), dtype=np.int64)
        lib().oracle_cones(self.h, level, box, step, _p(out, _lp), n)
        return out[:n]

    def grid(self, level, step):
        n = np.zeros(3, dtype=np.int64)
        lib().oracle_grid(self.h, level, step, _p(n, _lp))
        return n

    def orders(self, step):
        o = np.zeros(3, dtype=np.int32)
        lib().oracle_orders(self.h, step, _p(o, _ip))
        return o


def direct_sum(kind, k, srcs, w, tgts, tidx, normals=None, dx=-1):
    """FP64 dense sum u(y_t) = sum_s w_s G(x_s - y_t), Kahan-compensated."""
    kind = KINDS[kind] if isinstance(kind, str) else int(kind)
    k = complex(k)
    s = _aos(srcs)
    t = _aos(tgts)
    n = _aos(normals) if normals is not None else None
    w = np.ascontiguousarray(np.asarray(w, dtype=np.complex128))
    tidx = np.ascontiguousarray(np.asarray(tidx, dtype=np.int64))
    out = np.zeros(len(tidx), dtype=np.complex128)
    lib().oracle_direct(kind, k.real, k.imag, dx, _p(s), s.shape[0],
                        _p(n) if n is not None else None, _p(w.view(np.float64)), _p(t),
                        _p(tidx, _lp), len(tidx), _p(out.view(np.float64)))
    return out.real.copy() if kind == 0 else out


def dense_matrix(kind, k, srcs, tgts, normals=None, dx=-1):
    """The kernel matrix A[t, s] = G(x_s - y_t) that direct_sum applies
    (complex128, shape (M, N)); small cases only."""
    kind = KINDS[kind] if isinstance(kind, str) else int(kind)
    k = complex(k)
    s = _aos(srcs)
    t = _aos(tgts)
    n = _aos(normals) if normals is not None else None
    out = np.zeros((t.shape[0], s.shape[0]), dtype=np.complex128)
    lib().oracle_dense(kind, k.real, k.imag, dx, _p(s), s.shape[0],
                       _p(n) if n is not None else None, _p(t), t.shape[0],
                       _p(out.view(np.float64)))
    return out


def cheb_nodes(n):
    out = np.zeros(n)
    lib().oracle_cheb_nodes(n, _p(out))
    return out


def chebtransform3(ns, vals):
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    v = np.ascontiguousarray(vals, dtype=np.complex128)
    out = np.zeros_like(v)
    lib().oracle_chebtransform3(_p(ns, _ip), _p(v.view(np.float64)), _p(out.view(np.float64)))
    return out


def clenshaw3(ns, coef, x):
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    c = np.ascontiguousarray(coef, dtype=np.complex128)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(x.shape[0], dtype=np.complex128)
    lib().oracle_clenshaw3(_p(ns, _ip), _p(c.view(np.float64)), _p(x), x.shape[0],
                           _p(out.view(np.float64)))
    return out


def morton_less(bbmin, bbmax, p, q):
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (bbmin, bbmax, p, q)]
    return bool(lib().oracle_morton_less(*[_p(v) for v in a]))
