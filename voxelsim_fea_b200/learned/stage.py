"""Solver-side control of the learned stage (libvoxfea vf_learned_*).

The stage runs inside the solver's preconditioner -- z = V-cycle(r), then
z += P^L NN(R^L (r - A z)) -- and switches the iteration to flexible CG.
Weights are a flat FP32 vector in the libvoxfea layout (``UNet.flat_params``);
the trained set ships as ``unet_weights.npz`` next to this file.
"""

import ctypes
import os

import numpy as np

from .. import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "unet_weights.npz")


def param_count():
    return int(_lib.load().vf_learned_param_count())


def load_weights(path=WEIGHTS):
    """(params float32, level) of a saved network."""
    with np.load(path) as z:
        params = np.ascontiguousarray(z["params"], dtype=np.float32)
        level = int(z["level"])
    if params.size != param_count():
        raise ValueError(f"{path}: {params.size} parameters, the network has {param_count()}")
    return params, level


def save_weights(path, params, level, **meta):
    np.savez(path, params=np.asarray(params, dtype=np.float16), level=np.int32(level),
             **{k: np.asarray(v) for k, v in meta.items()})


def configure(solver, params=None, level=1, enable=True):
    """Create the stage on hierarchy level ``level`` of ``solver`` (an
    MGSolver), upload ``params`` when given, enable or disable it."""
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
    n = 0 if p is None else p.size
    _lib.check(_lib.load().vf_learned_configure(solver._handle(), int(level), _lib.ptr(p), n, int(bool(enable))),
               solver._h, "learned configure")


def enable_default(solver, path=WEIGHTS):
    params, level = load_weights(path)
    configure(solver, params, level, True)


def info(solver):
    d = (_lib._I32 * 3)()
    lv = _lib._I32()
    _lib.check(_lib.load().vf_learned_info(solver._handle(), d, ctypes.byref(lv)), solver._h, "learned info")
    return (int(d[0]), int(d[1]), int(d[2])), int(lv.value)


def level_mask(solver, level):
    lx, ly, lz = solver.levels[level]["dims"]
    out = np.empty((lx + 1) * (ly + 1) * (lz + 1), dtype=np.uint8)
    _lib.check(_lib.load().vf_level_mask(solver._handle(), int(level), out.ctypes.data_as(ctypes.c_void_p)),
               solver._h, "level mask")
    return out


def make_input(solver, r_level):
    """U-Net input of a level-L residual (host, reference node order of level
    L) as a (Z, Y, X, 16) BF16 CUDA tensor; returns (tensor, scale, eref)."""
    import torch
    (X, Y, Z), _ = info(solver)
    t = torch.empty((Z, Y, X, 16), device="cuda", dtype=torch.bfloat16)
    sc = ctypes.c_float()
    er = ctypes.c_double()
    r = _lib.f64(r_level)
    torch.cuda.synchronize()
    _lib.check(_lib.load().vf_learned_input(solver._handle(), _lib.ptr(r), ctypes.c_void_p(t.data_ptr()),
                                            ctypes.byref(sc), ctypes.byref(er)), solver._h, "learned input")
    return t, float(sc.value), float(er.value)


def apply(solver, r_fine):
    """The whole stage on a fine residual (host arrays): P^L NN(R^L r)."""
    out = np.empty(solver.ndof)
    r = _lib.f64(r_fine)
    _lib.check(_lib.load().vf_learned_apply(solver._handle(), _lib.ptr(r), _lib.ptr(out)), solver._h,
               "learned apply")
    return out
