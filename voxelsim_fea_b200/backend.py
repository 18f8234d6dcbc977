"""Compute-backend hook -- B200 edition.

Same module API as the reference's ``core/backend.py`` / ``core/backend_gpu.py``
(``is_gpu_build``, ``get_xp``, ``asnumpy``, ``gpu_usable``, ``gpu_device_count``,
``gpu_status``; core/backend_gpu.py:25-108), so callers that probe the backend
keep working.  The arrays callers see stay host numpy: device work happens
inside ``libvoxfea.so`` and the solve returns a fresh numpy array, exactly as
the reference returns ``xp.asnumpy(u)`` (core/multigrid.py:583).

``gpu_usable`` runs the library's self-test once (the hex8 operator on a small
grid, device vs host, core/backend_gpu.py:40-60 in spirit); unlike the
reference there is no silent CPU fallback: ``compute_plan.choose`` raises if
no usable device is present.
"""

import numpy as np

GPU_BUILD = True

_GPU_OK = None


def is_gpu_build():
    return GPU_BUILD


def get_xp(use_gpu=False):
    """Host array module of the API surface (numpy); kernels run in libvoxfea."""
    return np


def asnumpy(a):
    return np.asarray(a)


def _self_test():
    try:
        from . import _lib
        L = _lib.load()
        import ctypes
        n = ctypes.c_int32(0)
        if L.vf_device_count(ctypes.byref(n)) != 0 or n.value < 1:
            return False
        return L.vf_self_test(0) == 0
    except Exception:
        return False


def gpu_usable():
    """Cached: True only if libvoxfea loads, a device exists and the self-test passes."""
    global _GPU_OK
    if _GPU_OK is None:
        _GPU_OK = _self_test()
    return _GPU_OK


def gpu_device_count():
    try:
        from . import _lib
        import ctypes
        n = ctypes.c_int32(0)
        if _lib.load().vf_device_count(ctypes.byref(n)) != 0:
            return 0
        return int(n.value)
    except Exception:
        return 0


def gpu_status():
    try:
        from . import _lib
        _lib.load()
    except Exception as exc:  # noqa: BLE001
        return f"B200: libvoxfea unavailable ({exc})"
    if gpu_usable():
        return "B200: libvoxfea ready (self-test passed)"
    return "B200: no usable CUDA device / self-test failed"
