"""Operator classes with the reference's Python API (py_ifgf.cpp:16-58).

Each class mirrors one CRTP plug-in of the reference and keeps its
constructor arguments, ``init`` and ``mult``:

=====================================  ============================================
class                                  reference
=====================================  ============================================
LaplaceIfgfOperator                    laplace_ifgf.hpp, py_ifgf.cpp:45-48
HelmholtzIfgfOperator                  helmholtz_ifgf.hpp (not bound by py_ifgf)
ModifiedHelmholtzIfgfOperator          modified_helmholtz_ifgf.hpp, py_ifgf.cpp:37-38
  (alias MofifiedHelmholtzIfgfOperator, the reference's spelling)
GradHelmholtzIfgfOperator (+ setDx)    grad_helmholtz_ifgf.hpp, py_ifgf.cpp:39-40
DoubleLayerHelmholtzIfgfOperator       double_layer_helmholtz_ifgf.hpp
CombinedFieldHelmholtzIfgfOperator     combined_field_helmholtz_ifgf.hpp
=====================================  ============================================

Points are float64 arrays of shape (3, N).  ``mult`` takes a length-N
density (float64 for Laplace, complex128 otherwise) and returns the length-M
result in the caller's target order, like IfgfOperator::mult
(ifgfoperator.hpp:246-867).  Everything runs in libifgf_b200.so on the GPU.
"""
import ctypes as C
import json

import numpy as np

from . import _lib
from ._lib import check, lib


def _aos(pts, name):
    a = np.asarray(pts, dtype=np.float64)
    if a.ndim != 2 or a.shape[0] != 3:
        raise ValueError(f"{name} must have shape (3, N), got {a.shape}")
    return np.ascontiguousarray(a.T)


class IfgfOperator:
    """Common host logic of the IFGF operators (IfgfOperator, ifgfoperator.hpp:25-1936)."""

    KIND = None
    REAL = False
    NEEDS_NORMALS = False

    def __init__(self, k, leafSize, order, n_elem=1, tol=-1.0):
        k = complex(k)
        h = C.c_void_p()
        check(lib.ifgf_create(self.KIND, k.real, k.imag, int(leafSize), int(order), int(n_elem),
                              float(tol), C.byref(h)))
        self._h = h
        self._n_src = self._n_tgt = 0
        self.k = k

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.ifgf_destroy(h)
            self._h = None

    # -- setup --------------------------------------------------------------
    def _init(self, srcs, targets, normals=None, cutOff=None):
        s = _aos(srcs, "srcs")
        t = _aos(targets, "targets")
        n = None
        if self.NEEDS_NORMALS:
            if normals is None:
                raise ValueError("this operator needs source normals")
            n = _aos(normals, "normals")
            if n.shape != s.shape:
                raise ValueError("normals must have the same shape as srcs")
        cb = _lib.CUTOFF_FN(0)
        if cutOff is not None:
            def _cb(dist, _user, f=cutOff):
                return 1 if f(dist) else 0
            cb = _lib.CUTOFF_FN(_cb)
        dp = C.POINTER(C.c_double)
        # the library calls the cutoff again when it builds the adjoint's
        # operators, so the callback lives as long as the operator
        self._cutoff_cb = cb
        check(lib.ifgf_init(self._h, s.ctypes.data_as(dp), s.shape[0], t.ctypes.data_as(dp),
                            t.shape[0], n.ctypes.data_as(dp) if n is not None else None, cb, None))
        self._n_src, self._n_tgt = s.shape[0], t.shape[0]

    def init(self, srcs, targets, cutOff=None):
        """IfgfOperator::init (ifgfoperator.hpp:65-106)."""
        self._init(srcs, targets, None, cutOff)

    def init_plan_only(self, srcs, targets, cutOff=None):
        """Build the octrees and interaction lists on the host only (no GPU)."""
        s = _aos(srcs, "srcs")
        t = _aos(targets, "targets")
        cb = _lib.CUTOFF_FN(0)
        if cutOff is not None:
            def _cb(dist, _user, f=cutOff):
                return 1 if f(dist) else 0
            cb = _lib.CUTOFF_FN(_cb)
        dp = C.POINTER(C.c_double)
        check(lib.ifgf_init_plan_only(self._h, s.ctypes.data_as(dp), s.shape[0],
                                      t.ctypes.data_as(dp), t.shape[0], cb, None))
        self._n_src, self._n_tgt = s.shape[0], t.shape[0]

    def set_wavenumber(self, k):
        """Move the operator to wavenumber k (complex for the modified
        Helmholtz and gradient kernels), keeping the tree and cone maps when
        the cone grids allow (frequency sets)."""
        k = complex(k)
        check(lib.ifgf_set_wavenumber(self._h, k.real, k.imag))

    def set_shard(self, rank, nranks):
        """Take share `rank` of `nranks` of the matvec (call before init); the
        ranks' mult results sum to the full matvec (see ifgf_b200.distributed)."""
        check(lib.ifgf_set_shard(self._h, int(rank), int(nranks)))

    def shard_boxes(self):
        """(level, boxes): the shard level and this rank's boxes on it."""
        lev = C.c_int(0)
        n = C.c_long(0)
        check(lib.ifgf_shard_boxes(self._h, C.byref(lev), None, 0, C.byref(n)))
        out = np.zeros(n.value, dtype=np.int64)
        check(lib.ifgf_shard_boxes(self._h, C.byref(lev), out.ctypes.data_as(C.POINTER(C.c_long)),
                                   n.value, C.byref(n)))
        return lev.value, out

    def set_precision(self, mode):
        """"fp64" (default) or "mixed"."""
        m = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}.get(mode, mode)
        check(lib.ifgf_set_precision(self._h, int(m)))

    def set_upward_path(self, path):
        """Kernel of the mixed-precision upward transfer: "auto" (default;
        per level the faster of the two, timed on this operator), "ffma" or
        "tensor"."""
        p = {"auto": 0, "ffma": 1, "tensor": 2}.get(path, path)
        check(lib.ifgf_set_upward_path(self._h, int(p)))

    def set_far_plan(self, enable):
        """Far-field plan of the batched mixed matvecs: the far pairs' cone
        lookups done once and stored sorted by cone (default on; off frees
        its memory and looks the cones up in every matvec)."""
        check(lib.ifgf_set_far_plan(self._h, 1 if enable else 0))

    # -- matvec -------------------------------------------------------------
    def _dtype(self):
        return np.float64 if self.REAL else np.complex128

    def _out(self, out, shape):
        """The result array: a new one, or `out` when it fits (C-contiguous,
        the operator's dtype and the result's shape) -- e.g. pinned host
        memory, which the device-to-host copy then fills directly."""
        if out is None:
            return np.empty(shape, dtype=self._dtype())
        if (not isinstance(out, np.ndarray) or out.shape != shape or out.dtype != self._dtype()
                or not out.flags.c_contiguous):
            raise ValueError(f"out must be a C-contiguous {self._dtype().__name__} array of "
                             f"shape {shape}")
        return out

    def mult(self, weights, out=None):
        """IfgfOperator::mult (ifgfoperator.hpp:246-867)."""
        w = np.ascontiguousarray(np.asarray(weights, dtype=self._dtype()))
        if w.shape != (self._n_src,):
            raise ValueError(f"weights must have shape ({self._n_src},), got {w.shape}")
        u = self._out(out, (self._n_tgt,))
        check(lib.ifgf_mult(self._h, w.ctypes.data, u.ctypes.data))
        return u

    def mult_batch(self, weights, out=None):
        """A . w for every row of a (batch, N) array (into `out` when given)."""
        w = np.ascontiguousarray(np.asarray(weights, dtype=self._dtype()))
        if w.ndim != 2 or w.shape[1] != self._n_src:
            raise ValueError("weights must have shape (batch, N)")
        u = self._out(out, (w.shape[0], self._n_tgt))
        check(lib.ifgf_mult_batch(self._h, w.ctypes.data, u.ctypes.data, w.shape[0]))
        return u

    def mult_batch_device(self, w_ptr, u_ptr, batch, stream_ptr=0):
        """Enqueue A . w for `batch` right-hand sides on device buffers
        (batch x N in, batch x M out; raw pointers)."""
        check(lib.ifgf_mult_batch_device(self._h, C.c_void_p(w_ptr), C.c_void_p(u_ptr),
                                         int(batch), C.c_void_p(stream_ptr)))

    def mult_wavenumbers(self, ks, weights):
        """Row p of the result is A(k_p) . w_p, for wavenumbers ks (length L)
        and weights of shape (L, N); every k_p must give the operator's cone
        grids (a convolution-quadrature frequency set does).  The planes share
        one pass over the tree: one launch per stage and level for up to 64
        wavenumbers in mixed precision."""
        k = np.ascontiguousarray(np.asarray(ks, dtype=np.complex128).reshape(-1))
        w = np.ascontiguousarray(np.asarray(weights, dtype=self._dtype()))
        if w.ndim != 2 or w.shape != (k.size, self._n_src):
            raise ValueError(f"weights must have shape ({k.size}, {self._n_src})")
        u = np.empty((k.size, self._n_tgt), dtype=self._dtype())
        kd = k.view(np.float64)
        check(lib.ifgf_mult_wavenumbers(self._h, kd.ctypes.data_as(C.POINTER(C.c_double)),
                                        k.size, w.ctypes.data, u.ctypes.data))
        return u

    def mult_wavenumbers_device(self, ks, w_ptr, u_ptr, stream_ptr=0):
        """Enqueue mult_wavenumbers on device buffers (L x N in, L x M out;
        raw pointers)."""
        k = np.ascontiguousarray(np.asarray(ks, dtype=np.complex128).reshape(-1))
        kd = k.view(np.float64)
        check(lib.ifgf_mult_wavenumbers_device(self._h, kd.ctypes.data_as(C.POINTER(C.c_double)),
                                               k.size, C.c_void_p(w_ptr), C.c_void_p(u_ptr),
                                               C.c_void_p(stream_ptr)))

    def mult_device(self, w_ptr, u_ptr, stream_ptr=0):
        """Enqueue A . w on device buffers given as raw pointers (torch:
        tensor.data_ptr(), torch.cuda.current_stream().cuda_stream)."""
        check(lib.ifgf_mult_device(self._h, C.c_void_p(w_ptr), C.c_void_p(u_ptr),
                                   C.c_void_p(stream_ptr)))

    def mult_dk(self, weights):
        """(dA/dk) . w, the matvec of the wavenumber derivative of the kernel
        (Helmholtz and combined field); a (batch, N) array gives (batch, M)."""
        w = np.ascontiguousarray(np.asarray(weights, dtype=self._dtype()))
        batch = w.shape[0] if w.ndim == 2 else 1
        if w.shape[-1] != self._n_src or w.ndim > 2:
            raise ValueError(f"weights must have shape ([batch,] {self._n_src})")
        u = np.empty(w.shape[:-1] + (self._n_tgt,), dtype=self._dtype())
        check(lib.ifgf_mult_dk(self._h, w.ctypes.data, u.ctypes.data, batch))
        return u

    def mult_adjoint(self, weights):
        """A^H . w: one value per target in, one per source out; a (batch, M)
        array gives (batch, N)."""
        w = np.ascontiguousarray(np.asarray(weights, dtype=self._dtype()))
        batch = w.shape[0] if w.ndim == 2 else 1
        if w.shape[-1] != self._n_tgt or w.ndim > 2:
            raise ValueError(f"weights must have shape ([batch,] {self._n_tgt})")
        u = np.empty(w.shape[:-1] + (self._n_src,), dtype=self._dtype())
        check(lib.ifgf_mult_adjoint(self._h, w.ctypes.data, u.ctypes.data, batch))
        return u

    def mult_adjoint_device(self, w_ptr, u_ptr, stream_ptr=0):
        """Enqueue A^H . w on device buffers (raw pointers)."""
        check(lib.ifgf_mult_adjoint_device(self._h, C.c_void_p(w_ptr), C.c_void_p(u_ptr),
                                           C.c_void_p(stream_ptr)))

    def mult_dk_device(self, w_ptr, u_ptr, stream_ptr=0):
        """Enqueue (dA/dk) . w on device buffers (raw pointers)."""
        check(lib.ifgf_mult_dk_device(self._h, C.c_void_p(w_ptr), C.c_void_p(u_ptr),
                                      C.c_void_p(stream_ptr)))

    def direct_eval(self, weights, targets, dk=False):
        """FP64 dense direct sum at the given target indices (on the GPU);
        dk=True sums the k-derivative kernel."""
        w = np.ascontiguousarray(np.asarray(weights, dtype=self._dtype()))
        t = np.ascontiguousarray(np.asarray(targets, dtype=np.int64))
        out = np.empty(len(t), dtype=self._dtype())
        fn = lib.ifgf_direct_eval_dk if dk else lib.ifgf_direct_eval
        check(fn(self._h, w.ctypes.data, t.ctypes.data_as(C.POINTER(C.c_long)), len(t),
                 out.ctypes.data))
        return out

    def set_profiling(self, on=True):
        """Per-kernel CUDA-event timing of following mults (see stats()["profile"])."""
        check(lib.ifgf_set_profiling(self._h, 1 if on else 0))

    # -- introspection -------------------------------------------------------
    @property
    def n_src(self):
        return self._n_src

    @property
    def n_tgt(self):
        return self._n_tgt

    def stats(self):
        need = C.c_long(0)
        check(lib.ifgf_stats_json(self._h, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value)
        check(lib.ifgf_stats_json(self._h, buf, need.value, C.byref(need)))
        return json.loads(buf.value.decode())

    def levels(self, which=0):
        v = C.c_int(0)
        check(lib.ifgf_tree_levels(self._h, which, C.byref(v)))
        return v.value

    def num_boxes(self, level, which=0):
        v = C.c_long(0)
        check(lib.ifgf_tree_num_boxes(self._h, which, level, C.byref(v)))
        return v.value

    def permutation(self, which=0):
        n = self._n_src if which == 0 else self._n_tgt
        out = np.zeros(n, dtype=np.int64)
        check(lib.ifgf_tree_permutation(self._h, which, out.ctypes.data_as(C.POINTER(C.c_long))))
        return out

    def boxes(self, level, which=0):
        nb = self.num_boxes(level, which)
        ints = np.zeros((nb, 12), dtype=np.int64)
        bb = np.zeros((nb, 6), dtype=np.float64)
        check(lib.ifgf_tree_boxes(self._h, which, level, ints.ctypes.data_as(C.POINTER(C.c_long)),
                                  bb.ctypes.data_as(C.POINTER(C.c_double))))
        return ints, bb

    def interaction_list(self, level, box, far):
        n = C.c_long(0)
        check(lib.ifgf_box_list(self._h, level, box, int(far), None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 2), dtype=np.int64)
        check(lib.ifgf_box_list(self._h, level, box, int(far),
                                out.ctypes.data_as(C.POINTER(C.c_long)), n.value, C.byref(n)))
        return out[: n.value]

    def cones(self, level, box, step):
        n = C.c_long(0)
        check(lib.ifgf_box_cones(self._h, level, box, step, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), dtype=np.int64)
        check(lib.ifgf_box_cones(self._h, level, box, step,
                                 out.ctypes.data_as(C.POINTER(C.c_long)), n.value, C.byref(n)))
        return out[: n.value]

    def grid(self, level, step):
        n = np.zeros(3, dtype=np.int64)
        check(lib.ifgf_level_grid(self._h, level, step, n.ctypes.data_as(C.POINTER(C.c_long))))
        return n

    def orders(self, step):
        o = np.zeros(3, dtype=np.int32)
        check(lib.ifgf_orders(self._h, step, o.ctypes.data_as(C.POINTER(C.c_int))))
        return o


class LaplaceIfgfOperator(IfgfOperator):
    """1/(4 pi r) (laplace_ifgf.hpp); T = float64."""

    KIND = _lib.LAPLACE
    REAL = True

    def __init__(self, leafSize, order, n_elem=1, tol=-1.0):
        super().__init__(0.0, leafSize, order, n_elem, tol)


class HelmholtzIfgfOperator(IfgfOperator):
    """e^{ikr}/(4 pi r), real k (helmholtz_ifgf.hpp)."""

    KIND = _lib.HELMHOLTZ

    def __init__(self, waveNumber, leafSize, order, n_elem=1, tol=-1.0):
        super().__init__(float(np.real(waveNumber)), leafSize, order, n_elem, tol)


class ModifiedHelmholtzIfgfOperator(IfgfOperator):
    """e^{-kr}/(4 pi r), complex k (modified_helmholtz_ifgf.hpp)."""

    KIND = _lib.MODIFIED_HELMHOLTZ


# the reference's Python name (py_ifgf.cpp:37-38), spelling kept
MofifiedHelmholtzIfgfOperator = ModifiedHelmholtzIfgfOperator


class GradHelmholtzIfgfOperator(IfgfOperator):
    """d/dy_dx e^{-k|x-y|}/(4 pi |x-y|) (grad_helmholtz_ifgf.hpp); setDx(-1)
    selects the plain single layer."""

    KIND = _lib.GRAD_HELMHOLTZ

    def setDx(self, dx):
        check(lib.ifgf_set_dx(self._h, int(dx)))


class DoubleLayerHelmholtzIfgfOperator(IfgfOperator):
    """Double layer with source normals (double_layer_helmholtz_ifgf.hpp)."""

    KIND = _lib.DOUBLE_LAYER
    NEEDS_NORMALS = True

    def init(self, srcs, targets, normals, cutOff=None):
        self._init(srcs, targets, normals, cutOff)


class CombinedFieldHelmholtzIfgfOperator(IfgfOperator):
    """Double layer minus i kappa single layer, real kappa
    (combined_field_helmholtz_ifgf.hpp)."""

    KIND = _lib.COMBINED_FIELD
    NEEDS_NORMALS = True

    def __init__(self, waveNumber, leafSize, order, n_elem=1, tol=-1.0):
        super().__init__(float(np.real(waveNumber)), leafSize, order, n_elem, tol)

    def init(self, srcs, targets, normals, cutOff=None):
        self._init(srcs, targets, normals, cutOff)
