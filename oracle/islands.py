"""Support-connectivity pre-step (oracle, test-only).

Restates VoxelSim-FEA ``core/fea.py:151-227``: elements that are not
6-connected (through face-adjacent active elements) to an element touching a
fixed node are dropped before the solve.
"""

import numpy as np

from .hex8 import build_edof


def seed_from_fixed_dofs(nx, ny, nz, fixed_dofs):
    """(nx,ny,nz) bool: elements touching >= 1 fixed node (fea.py:165-177)."""
    n_nodes = (nx + 1) * (ny + 1) * (nz + 1)
    fixed_dofs = np.asarray(fixed_dofs, dtype=np.int64)
    if fixed_dofs.size == 0:
        return np.zeros((nx, ny, nz), dtype=bool)
    is_fixed = np.zeros(n_nodes, dtype=bool)
    is_fixed[np.unique(fixed_dofs // 3)] = True
    node_ids = build_edof(nx, ny, nz)[:, 0::3] // 3
    return is_fixed[node_ids].any(axis=1).reshape(nx, ny, nz)


def connected_component_mask(active3d, seed3d):
    """6-connected iterative dilation flood fill (fea.py:180-204)."""
    active3d = np.asarray(active3d, dtype=bool)
    reached = np.asarray(seed3d, dtype=bool) & active3d
    if not reached.any():
        return reached
    while True:
        grown = reached.copy()
        grown[1:, :, :] |= reached[:-1, :, :]
        grown[:-1, :, :] |= reached[1:, :, :]
        grown[:, 1:, :] |= reached[:, :-1, :]
        grown[:, :-1, :] |= reached[:, 1:, :]
        grown[:, :, 1:] |= reached[:, :, :-1]
        grown[:, :, :-1] |= reached[:, :, 1:]
        grown &= active3d
        if np.array_equal(grown, reached):
            return reached
        reached = grown


def drop_unsupported_islands(active3d, fixed_dofs):
    """(kept3d, n_removed); input returned unchanged when nothing is reached
    (fea.py:207-227)."""
    active3d = np.asarray(active3d, dtype=bool)
    nx, ny, nz = active3d.shape
    kept = connected_component_mask(active3d,
                                     seed_from_fixed_dofs(nx, ny, nz, fixed_dofs))
    if not kept.any():
        return active3d, 0
    return kept, int(active3d.sum() - kept.sum())
