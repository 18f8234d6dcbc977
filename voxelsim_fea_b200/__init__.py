"""B200-native matrix-free voxel elasticity solve (hex8 GMG-PCG).

Drop-in for VoxelSim-FEA's solver layer (``core/fea.py``, ``core/multigrid.py``,
``core/compute_plan.py``, ``core/backend*.py``): same classes, signatures,
attributes and error behaviour, computing on sm_100a through the C-ABI library
``libvoxfea.so`` (declared in ``include/voxfea.h``).

Importing this package does not touch the GPU; constructing a solver loads the
library and raises if it (or a CUDA device) is missing -- there is no CPU path.
"""

__all__ = ["MGSolver", "VoxelFEA", "compute_plan", "backend", "generators"]

from . import backend, compute_plan, generators  # noqa: E402


def __getattr__(name):
    if name == "MGSolver":
        from .multigrid import MGSolver
        return MGSolver
    if name == "VoxelFEA":
        from .fea import VoxelFEA
        return VoxelFEA
    raise AttributeError(name)
