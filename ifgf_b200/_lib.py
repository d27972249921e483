"""ctypes binding of libifgf_b200.so (the C ABI in include/ifgf_b200.h).

The CUDA library is the only implementation: importing this module fails
loudly when the shared library has not been built.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libifgf_b200.so")

IFGF_OK = 0
ERRORS = {
    1: "invalid argument",
    2: "CUDA error",
    3: "invalid state",
    4: "out of memory",
    5: "device wait timed out",
    6: "internal error",
}

LAPLACE, HELMHOLTZ, MODIFIED_HELMHOLTZ, GRAD_HELMHOLTZ, DOUBLE_LAYER, COMBINED_FIELD = range(6)
PREC_FP64, PREC_MIXED = 0, 1

CUTOFF_FN = C.CFUNCTYPE(C.c_int, C.c_double, C.c_void_p)

_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_long)
_ip = C.POINTER(C.c_int)


class IfgfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python -c 'import __graft_entry__ as g; g.build()' or python ifgf_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    H = C.c_void_p
    sig = {
        "ifgf_create": [C.c_int, C.c_double, C.c_double, C.c_long, C.c_long, C.c_long, C.c_double,
                        C.POINTER(H)],
        "ifgf_set_dx": [H, C.c_int],
        "ifgf_set_precision": [H, C.c_int],
        "ifgf_set_upward_path": [H, C.c_int],
        "ifgf_set_far_plan": [H, C.c_int],
        "ifgf_bounded_wait_selftest": [C.c_double, _dp],
        "ifgf_set_shard": [H, C.c_int, C.c_int],
        "ifgf_set_wavenumber": [H, C.c_double, C.c_double],
        "ifgf_shard_boxes": [H, _ip, _lp, C.c_long, _lp],
        "ifgf_init": [H, _dp, C.c_long, _dp, C.c_long, _dp, CUTOFF_FN, C.c_void_p],
        "ifgf_init_plan_only": [H, _dp, C.c_long, _dp, C.c_long, CUTOFF_FN, C.c_void_p],
        "ifgf_box_list": [H, C.c_int, C.c_long, C.c_int, _lp, C.c_long, _lp],
        "ifgf_mult": [H, C.c_void_p, C.c_void_p],
        "ifgf_mult_batch": [H, C.c_void_p, C.c_void_p, C.c_long],
        "ifgf_mult_device": [H, C.c_void_p, C.c_void_p, C.c_void_p],
        "ifgf_mult_batch_device": [H, C.c_void_p, C.c_void_p, C.c_long, C.c_void_p],
        "ifgf_mult_device_noalloc": [H, C.c_void_p, C.c_void_p, C.c_void_p],
        "ifgf_mult_wavenumbers": [H, _dp, C.c_long, C.c_void_p, C.c_void_p],
        "ifgf_mult_wavenumbers_device": [H, _dp, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p],
        "ifgf_direct_eval": [H, C.c_void_p, _lp, C.c_long, C.c_void_p],
        "ifgf_direct_eval_dk": [H, C.c_void_p, _lp, C.c_long, C.c_void_p],
        "ifgf_mult_dk": [H, C.c_void_p, C.c_void_p, C.c_long],
        "ifgf_mult_adjoint": [H, C.c_void_p, C.c_void_p, C.c_long],
        "ifgf_mult_adjoint_device": [H, C.c_void_p, C.c_void_p, C.c_void_p],
        "ifgf_mult_dk_device": [H, C.c_void_p, C.c_void_p, C.c_void_p],
        "ifgf_set_profiling": [H, C.c_int],
        "ifgf_num_sources": [H, _lp],
        "ifgf_num_targets": [H, _lp],
        "ifgf_stats_json": [H, C.c_char_p, C.c_long, _lp],
        "ifgf_tree_levels": [H, C.c_int, _ip],
        "ifgf_tree_num_boxes": [H, C.c_int, C.c_int, _lp],
        "ifgf_tree_permutation": [H, C.c_int, _lp],
        "ifgf_tree_boxes": [H, C.c_int, C.c_int, _lp, _dp],
        "ifgf_box_cones": [H, C.c_int, C.c_long, C.c_int, _lp, C.c_long, _lp],
        "ifgf_level_grid": [H, C.c_int, C.c_int, _lp],
        "ifgf_orders": [H, C.c_int, _ip],
        "ifgf_destroy": [H],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.ifgf_last_error.argtypes = []
    L.ifgf_last_error.restype = C.c_char_p
    return L


lib = _load()

# Every symbol declared in include/ifgf_b200.h.
EXPORTED = [
    "ifgf_create", "ifgf_set_dx", "ifgf_set_precision", "ifgf_set_shard", "ifgf_shard_boxes",
    "ifgf_set_upward_path", "ifgf_set_far_plan", "ifgf_bounded_wait_selftest",
    "ifgf_set_wavenumber",
    "ifgf_init", "ifgf_init_plan_only",
    "ifgf_box_list", "ifgf_mult",
    "ifgf_mult_batch", "ifgf_mult_batch_device", "ifgf_mult_device", "ifgf_mult_device_noalloc",
    "ifgf_mult_wavenumbers", "ifgf_mult_wavenumbers_device",
    "ifgf_direct_eval",
    "ifgf_mult_dk", "ifgf_mult_dk_device", "ifgf_direct_eval_dk", "ifgf_mult_adjoint",
    "ifgf_mult_adjoint_device",
    "ifgf_set_profiling",
    "ifgf_num_sources", "ifgf_num_targets",
    "ifgf_stats_json", "ifgf_tree_levels", "ifgf_tree_num_boxes", "ifgf_tree_permutation",
    "ifgf_tree_boxes", "ifgf_box_cones", "ifgf_level_grid", "ifgf_orders", "ifgf_destroy",
    "ifgf_last_error",
]


def check(code):
    if code != IFGF_OK:
        raise IfgfError(code, lib.ifgf_last_error().decode())
