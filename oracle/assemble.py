"""Grid assembly of a solve job (oracle, test-only): a numpy restatement of
the reference worker's role-mask bookkeeping (core/solve_worker.py:242-270).

The last ``build`` mask is the active set, ``exclude`` masks are removed from
it; every ``bearing`` mask fixes the flagged axes of its nodes; every ``load``
mask spreads its force evenly over its nodes, role by role in job order."""

import numpy as np


def assemble(descr, masks, dims):
    """(active bool[nelem], fixed_dofs int64 sorted unique, force float64[ndof])."""
    nx, ny, nz = dims
    inside = None
    excl = np.zeros(nx * ny * nz, dtype=bool)
    fixed = []
    force = np.zeros(3 * (nx + 1) * (ny + 1) * (nz + 1))
    for (role, meta), mask in zip(descr, masks):
        mask = np.asarray(mask, dtype=bool)
        if role == "build":                          # solve_worker.py:250-251
            inside = mask
        elif role == "exclude":                      # :252-253
            excl = excl | mask
        elif role == "bearing":                      # :254-262
            nodes = np.nonzero(mask)[0]
            for c, on in enumerate(meta):
                if on:
                    fixed.append(3 * nodes + c)
        elif role == "load":                         # :263-268
            nodes = np.nonzero(mask)[0]
            if len(nodes):
                fv = np.asarray(meta, dtype=float) / len(nodes)
                for c in range(3):
                    force[3 * nodes + c] += fv[c]
    if inside is None:
        inside = np.zeros(nx * ny * nz, dtype=bool)
    active = inside & ~excl
    fixed_dofs = np.unique(np.concatenate(fixed)).astype(np.int64) if fixed else np.zeros(0, dtype=np.int64)
    return active, fixed_dofs, force
