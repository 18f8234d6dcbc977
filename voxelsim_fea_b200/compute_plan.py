"""Compute-backend selection -- B200 edition.

Keeps the reference's module surface (``ComputePlan``, ``cpu_worker_count``,
``configure_cpu_threads``, ``choose``, the DOF thresholds;
core/compute_plan.py:51-194) and adds the plan kind ``"b200"``: the single
device path of this package.  Every request resolves to it -- the reference's
CPU / multi-process / multi-GPU tiers are not rebuilt (one device, no
sharding, no CPU fallback) -- and ``choose`` raises when no usable device is
present instead of degrading silently.
"""

import os

from . import backend

GPU_DOF = 50_000
MULTI_GPU_DOF = 50_000_000
MULTI_CPU_DOF = 500_000
VALID_MODES = ("AUTO", "CPU", "GPU", "MULTI_GPU", "MULTI_CPU", "B200")

_THREADPOOL_LIMITER = None


class ComputePlan:
    """Resolved decision for one solver instance (core/compute_plan.py:62-77)."""

    __slots__ = ("kind", "xp", "n_workers", "label")

    def __init__(self, kind, xp, n_workers, label):
        self.kind = kind
        self.xp = xp
        self.n_workers = n_workers
        self.label = label

    @property
    def parallel(self):
        return self.kind in ("multi_gpu", "multi_cpu")


def cpu_worker_count(requested=0):
    """All logical cores minus one unless a positive count is requested
    (core/compute_plan.py:80-90)."""
    total = os.cpu_count() or 1
    if requested and requested > 0:
        return max(1, min(int(requested), total))
    return max(1, total - 1)


def configure_cpu_threads(n_threads, verbose=False):
    """Limit the host BLAS pool (core/compute_plan.py:93-125); no-op without
    threadpoolctl.  Host BLAS is not on the solve path here."""
    global _THREADPOOL_LIMITER
    try:
        import threadpoolctl
    except Exception:
        return None
    try:
        if _THREADPOOL_LIMITER is not None:
            _THREADPOOL_LIMITER.unregister()
        _THREADPOOL_LIMITER = threadpoolctl.threadpool_limits(limits=int(n_threads))
        return _THREADPOOL_LIMITER
    except Exception:
        return None


def choose(ndof, mode="AUTO", cpu_threads=0, verbose=False):
    """Resolve the plan for ``ndof`` DOFs: always the B200 device path."""
    mode = (mode or "AUTO").upper()
    if mode not in VALID_MODES:
        raise ValueError(f"unknown compute_mode {mode!r}; expected one of {VALID_MODES}")
    if not backend.gpu_usable():
        raise RuntimeError(
            "no usable sm_100 device for libvoxfea (this build has no CPU path): "
            + backend.gpu_status())
    label = "B200 (sm_100a, libvoxfea)"
    if mode not in ("AUTO", "GPU", "B200"):
        label += f" [requested {mode}; single-device path]"
    plan = ComputePlan("b200", backend.get_xp(True), 1, label)
    if verbose:
        print(f"[VoxelSim FEA] compute plan: ndof={ndof} mode={mode} -> {plan.label}")
    return plan
