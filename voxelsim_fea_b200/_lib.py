"""ctypes binding of libvoxfea.so (the C-ABI declared in include/voxfea.h).

The library is built in-tree (``python -m voxelsim_fea_b200.build``) and loaded
from this package directory.  There is no fallback: if the shared library or
a CUDA device is missing, loading raises.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvoxfea.so")

VF_OK = 0
VF_ERR_ARG = 1
VF_ERR_STATE = 2
VF_ERR_CUDA = 3
VF_ERR_NOMEM = 4
VF_ERR_NO_DEVICE = 5
VF_ERR_STALLED = 6
VF_ERR_NONFINITE = 7
VF_ERR_UNSUPPORTED = 8
VF_ERR_BREAKDOWN = 9

VF_PREC_FP64, VF_PREC_MIXED, VF_PREC_FP32 = 0, 1, 2
VF_METHOD_MG, VF_METHOD_JACOBI = 0, 1
VF_COARSE_REDISCRETIZE, VF_COARSE_GALERKIN = 0, 1
VF_COARSEST_JACOBI, VF_COARSEST_CHOLESKY = 0, 1
VF_SOLVE_DEVICE_PTRS = 1
VF_OMEGA_FIXED, VF_OMEGA_AUTO = 0, 1
VF_FINE_MODAL, VF_FINE_GATHER, VF_FINE_MODAL_CPASYNC = 0, 1, 2
STENCIL_STORAGE = {"sym_half": 0, "sym": 1, "full": 2}
MIXED_MODES = {"reliable": 0, "restart": 1, "outer64": 2}
SMOOTHERS = {"jacobi": 0, "chebyshev": 1}
ROLES = {"build": 0, "exclude": 1, "bearing": 2, "load": 3}   # VF_ROLE_* of vf_assemble_grid

PRECISIONS = {"fp64": VF_PREC_FP64, "mixed": VF_PREC_MIXED, "fp32": VF_PREC_FP32}
COARSE_OPS = {"rediscretize": VF_COARSE_REDISCRETIZE, "galerkin": VF_COARSE_GALERKIN}
COARSEST = {"jacobi": VF_COARSEST_JACOBI, "cholesky": VF_COARSEST_CHOLESKY}

# every symbol include/voxfea.h declares (checked by the CPU test suite)
EXPORTS = (
    "vf_abi_version", "vf_status_string", "vf_global_last_error", "vf_device_count",
    "vf_self_test", "vf_hex8_tables", "vf_options_default", "vf_create", "vf_destroy", "vf_last_error",
    "vf_num_levels", "vf_level_dims", "vf_level_omega", "vf_set_fixed", "vf_set_active", "vf_set_material",
    "vf_solve", "vf_solve_cb", "vf_resid_history", "vf_von_mises", "vf_strain_energy",
    "vf_drop_unsupported_islands", "vf_apply", "vf_smooth", "vf_restrict", "vf_prolongate",
    "vf_vcycle", "vf_inv_diagonal", "vf_time_kernel", "vf_get_stream", "vf_launch_count",
    "vf_apply_noalloc",
    "vf_nn_conv3d_forward", "vf_nn_conv3d_backward_data", "vf_nn_conv3d_backward_weight",
    "vf_nn_wgrad_workspace", "vf_learned_param_count", "vf_learned_configure", "vf_learned_info",
    "vf_learned_input", "vf_learned_apply", "vf_level_mask", "vf_mg_propagate", "vf_solve_block",
    "vf_solve_batch", "vf_inside_points", "vf_inside_grid", "vf_element_displacement",
    "vf_assemble_grid", "vf_drop_unsupported_islands_mask", "vf_set_fixed_mask",
)


class VfOptions(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("method", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("n_smooth", ctypes.c_int32),
        ("min_elems", ctypes.c_int32), ("max_levels", ctypes.c_int32),
        ("coarse_op", ctypes.c_int32), ("coarsest", ctypes.c_int32),
        ("coarse_sweeps", ctypes.c_int32), ("stall_guard", ctypes.c_int32),
        ("check_every", ctypes.c_int32), ("use_graphs", ctypes.c_int32),
        ("device", ctypes.c_int32), ("max_outer", ctypes.c_int32),
        ("omega", ctypes.c_double), ("inner_tol", ctypes.c_double),
        ("omega_mode", ctypes.c_int32), ("power_iters", ctypes.c_int32),
        ("omega_rel", ctypes.c_double),
        ("fine_kernel", ctypes.c_int32), ("modal_zchunk", ctypes.c_int32),
        ("coarse_storage", ctypes.c_int32), ("mixed_mode", ctypes.c_int32),
        ("flexible", ctypes.c_int32), ("autotune", ctypes.c_int32),
        ("smoother", ctypes.c_int32), ("cheb_ratio", ctypes.c_int32),
        ("smoothed_transfers", ctypes.c_int32), ("learned_watch", ctypes.c_int32),
        ("smoothed_level_sweeps", ctypes.c_int32),
    ]


class VfSolveInfo(ctypes.Structure):
    _fields_ = [
        ("iters", ctypes.c_int32), ("outer_iters", ctypes.c_int32),
        ("converged", ctypes.c_int32), ("status", ctypes.c_int32),
        ("resid_ratio", ctypes.c_double), ("true_resid", ctypes.c_double),
        ("device_ms", ctypes.c_double), ("setup_ms", ctypes.c_double),
    ]


PROGRESS_FN = ctypes.CFUNCTYPE(None, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_void_p)

_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I32 = ctypes.c_int32
_lib = None


class LibraryMissing(RuntimeError):
    pass


class StallError(RuntimeError):
    """The MG-PCG stall/divergence guard fired (core/multigrid.py:523-531)."""


def _declare(L):
    sig = {
        "vf_abi_version": (ctypes.c_int, []),
        "vf_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "vf_global_last_error": (ctypes.c_char_p, []),
        "vf_device_count": (ctypes.c_int, [ctypes.POINTER(_I32)]),
        "vf_self_test": (ctypes.c_int, [_I32]),
        "vf_hex8_tables": (ctypes.c_int, [ctypes.c_double, _P, _P, _P, _P]),
        "vf_options_default": (None, [ctypes.POINTER(VfOptions)]),
        "vf_create": (ctypes.c_int, [_I32, _I32, _I32, ctypes.c_double, ctypes.POINTER(VfOptions),
                                     ctypes.POINTER(_P)]),
        "vf_destroy": (ctypes.c_int, [_P]),
        "vf_last_error": (ctypes.c_char_p, [_P]),
        "vf_num_levels": (ctypes.c_int, [_P, ctypes.POINTER(_I32)]),
        "vf_level_dims": (ctypes.c_int, [_P, _I32, ctypes.POINTER(_I32)]),
        "vf_level_omega": (ctypes.c_int, [_P, _I32, _D, _D]),
        "vf_set_fixed": (ctypes.c_int, [_P, _P, ctypes.c_int64]),
        "vf_set_active": (ctypes.c_int, [_P, _P]),
        "vf_set_material": (ctypes.c_int, [_P, _P, _P, ctypes.c_uint32]),
        "vf_solve": (ctypes.c_int, [_P, _P, _P, ctypes.c_double, _I32, ctypes.c_uint32, _P,
                                    ctypes.POINTER(VfSolveInfo)]),
        "vf_solve_cb": (ctypes.c_int, [_P, _P, _P, ctypes.c_double, _I32, ctypes.c_uint32, _P,
                                       ctypes.POINTER(VfSolveInfo), PROGRESS_FN, _P]),
        "vf_resid_history": (ctypes.c_int, [_P, _P, _I32, ctypes.POINTER(_I32)]),
        "vf_von_mises": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
        "vf_strain_energy": (ctypes.c_int, [_P, _P, _P, _P]),
        "vf_drop_unsupported_islands": (ctypes.c_int, [_I32, _I32, _I32, _P, _P, ctypes.c_int64, _P,
                                                       ctypes.POINTER(ctypes.c_int64)]),
        "vf_apply": (ctypes.c_int, [_P, _I32, _I32, _P, _P]),
        "vf_smooth": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _I32, _P]),
        "vf_restrict": (ctypes.c_int, [_P, _I32, _I32, _P, _P]),
        "vf_prolongate": (ctypes.c_int, [_P, _I32, _I32, _P, _P]),
        "vf_vcycle": (ctypes.c_int, [_P, _I32, _P, _P]),
        "vf_inv_diagonal": (ctypes.c_int, [_P, _I32, _P]),
        "vf_time_kernel": (ctypes.c_int, [_P, _I32, _I32, _I32, _D]),
        "vf_get_stream": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_void_p)]),
        "vf_launch_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint64)]),
        "vf_apply_noalloc": (ctypes.c_int, [_I32, _I32, _I32, ctypes.c_double, _P, _P, _P, _P, _P, _P]),
        "vf_nn_conv3d_forward": (ctypes.c_int, [_P, _P, _P, _P, _I32, _P, _P, _I32, _I32, _I32, _I32, _I32, _P]),
        "vf_nn_conv3d_backward_data": (ctypes.c_int, [_P, _P, _P, _P, _I32, _I32, _I32, _I32, _I32, _P]),
        "vf_nn_conv3d_backward_weight": (ctypes.c_int, [_P, _P, _P, _I32, _P, ctypes.c_size_t, _I32, _I32, _I32,
                                                        _I32, _I32, _P]),
        "vf_nn_wgrad_workspace": (ctypes.c_size_t, [_I32, _I32, _I32, _I32, _I32]),
        "vf_learned_param_count": (ctypes.c_int64, []),
        "vf_learned_configure": (ctypes.c_int, [_P, _I32, _P, ctypes.c_int64, _I32]),
        "vf_learned_info": (ctypes.c_int, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
        "vf_learned_input": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(ctypes.c_float), _D]),
        "vf_learned_apply": (ctypes.c_int, [_P, _P, _P]),
        "vf_level_mask": (ctypes.c_int, [_P, _I32, _P]),
        "vf_mg_propagate": (ctypes.c_int, [_P, _P, _I32, _P]),
        "vf_solve_block": (ctypes.c_int, [_P, _P, _I32, ctypes.c_double, _I32, ctypes.c_uint32, _P,
                                          ctypes.POINTER(VfSolveInfo)]),
        "vf_solve_batch": (ctypes.c_int, [_P, _I32, _P, _P, _P, ctypes.c_double, _I32, ctypes.c_uint32, _P,
                                          ctypes.POINTER(VfSolveInfo)]),
        "vf_inside_points": (ctypes.c_int, [_P, ctypes.c_int64, _P, ctypes.c_int64, _P, ctypes.c_int64, _P, _P]),
        "vf_element_displacement": (ctypes.c_int, [_I32, _I32, _I32, _P, _P]),
        "vf_assemble_grid": (ctypes.c_int, [_I32, _I32, _I32, _I32, _P, _P, _P, ctypes.c_uint32, _P, _P, _P,
                                            ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
        "vf_drop_unsupported_islands_mask": (ctypes.c_int, [_I32, _I32, _I32, _P, _P, ctypes.c_uint32, _P,
                                                            ctypes.POINTER(ctypes.c_int64)]),
        "vf_set_fixed_mask": (ctypes.c_int, [_P, _P, ctypes.c_uint32]),
        "vf_inside_grid": (ctypes.c_int, [_P, ctypes.c_int64, _P, ctypes.c_int64, _P, _P, ctypes.c_double, _I32,
                                          _P, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def load(path=LIB_PATH):
    """Load (once) and return the library handle; raises LibraryMissing."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise LibraryMissing(
                f"{path} is not built; run `python -m voxelsim_fea_b200.build` "
                "(this package has no CPU fallback)")
        L = ctypes.CDLL(path)
        _declare(L)
        _lib = L
    return _lib


def default_options():
    o = VfOptions()
    load().vf_options_default(ctypes.byref(o))
    return o


def ptr(a):
    """Raw pointer of a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def check(rc, handle=None, what=""):
    """Map a status code to the reference's exception types."""
    if rc == VF_OK:
        return
    L = load()
    msg = ""
    if handle is not None:
        msg = (L.vf_last_error(handle) or b"").decode(errors="replace")
    if not msg:
        msg = (L.vf_global_last_error() or b"").decode(errors="replace")
    text = f"{what}: {L.vf_status_string(rc).decode()} ({msg})" if what else \
        f"{L.vf_status_string(rc).decode()} ({msg})"
    if rc == VF_ERR_ARG:
        raise ValueError(text)
    if rc == VF_ERR_NOMEM:
        raise MemoryError(text)
    if rc == VF_ERR_NONFINITE:
        raise FloatingPointError(text)
    if rc == VF_ERR_UNSUPPORTED:
        raise NotImplementedError(text)
    if rc == VF_ERR_STALLED:
        raise StallError(msg or text)
    if rc == VF_ERR_STATE:
        raise RuntimeError(msg or text)
    raise RuntimeError(text)
