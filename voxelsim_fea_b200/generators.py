"""Seeded synthetic voxel problems (inputs for benchmarks and parity tests).

Every problem is a plain dict in the reference solver's own conventions
(VoxelSim-FEA ``core/solve_worker.py:242-358``):

* ``active``      bool (nelem,), element order iz-fastest (``build_edof``)
* ``E_stiff``     float64 (nelem,) = E * vsize, the stiffness modulus passed to
                  ``solve`` (solve_worker.py:354)
* ``E_stress``    float64 (nelem,) = E, for von Mises (solve_worker.py:355)
* ``nu``          scalar Poisson ratio, or float64 (nelem,) for two materials
* ``fixed_dofs``  int64 sorted unique global DOF ids (3*node + c)
* ``f``           float64 (3*(nx+1)*(ny+1)*(nz+1),) nodal forces, a load's total
                  spread evenly over its nodes (solve_worker.py:262-267)

Geometry generators use numpy + scipy.ndimage (Gaussian blur, 26-connected
labelling); no dataset is involved, all inputs are reproducible from the seed.
"""

import numpy as np

STEEL = (200e9, 0.30)
ALUMINUM = (69e9, 0.33)
ABS = (2.3e9, 0.35)


def _node_ids_of_elements(ex, ey, ez, nx, ny):
    """(n, 8) node ids of elements (reference local corner order)."""
    offs = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
            (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))
    out = np.empty((np.size(ex), 8), dtype=np.int64)
    for k, (ox, oy, oz) in enumerate(offs):
        out[:, k] = (ex + ox) + (nx + 1) * ((ey + oy) + (ny + 1) * (ez + oz))
    return out


def _dofs_of_nodes(nodes, comps=(0, 1, 2)):
    nodes = np.unique(np.asarray(nodes, dtype=np.int64))
    return np.unique(np.concatenate([3 * nodes + c for c in comps])) if nodes.size else \
        np.zeros(0, dtype=np.int64)


def cantilever(nx=64, ny=16, nz=16, vsize=1e-3, material=STEEL, load_n=1000.0):
    """Solid beam, x=0 face clamped on XYZ, total ``load_n`` in -z spread over
    the x=max face nodes."""
    E, nu = material
    nelem = nx * ny * nz
    n_nodes = (nx + 1) * (ny + 1) * (nz + 1)
    iy, iz = np.meshgrid(np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    face0 = (0 + (nx + 1) * (iy + (ny + 1) * iz)).ravel()
    face1 = (nx + (nx + 1) * (iy + (ny + 1) * iz)).ravel()
    f = np.zeros(3 * n_nodes)
    f[3 * face1 + 2] = -load_n / face1.size
    return {
        "name": f"cantilever_{nx}x{ny}x{nz}", "dims": (nx, ny, nz), "vsize": vsize,
        "active": np.ones(nelem, dtype=bool),
        "E_stiff": np.full(nelem, E * vsize), "E_stress": np.full(nelem, E),
        "nu": nu, "fixed_dofs": _dofs_of_nodes(face0), "f": f,
    }


def _blurred_noise(rng, shape, sigma):
    from scipy import ndimage
    return ndimage.gaussian_filter(rng.standard_normal(shape), sigma=sigma, mode="reflect")


def noise_solid(shape, seed, sigma=4.0, fill_percentile=50.0):
    """Blurred Gaussian noise thresholded at a percentile; largest
    26-connected component kept. Returns bool (nx, ny, nz)."""
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    field = _blurred_noise(rng, shape, sigma)
    solid = field > np.percentile(field, fill_percentile)
    lab, n = ndimage.label(solid, structure=np.ones((3, 3, 3), dtype=bool))
    if n == 0:
        return solid
    sizes = np.bincount(lab.ravel())
    sizes[0] = 0
    return lab == int(np.argmax(sizes))


def _top_patch_nodes(solid3d, cx, cy, half_w, half_h):
    """Nodes of the top face of the highest solid voxel in every column of the
    patch [cx-half_w, cx+half_w) x [cy-half_h, cy+half_h)."""
    nx, ny, nz = solid3d.shape
    nodes = []
    for ix in range(max(cx - half_w, 0), min(cx + half_w, nx)):
        for iy in range(max(cy - half_h, 0), min(cy + half_h, ny)):
            col = np.nonzero(solid3d[ix, iy, :])[0]
            if col.size == 0:
                continue
            top = int(col[-1]) + 1
            for ox in (0, 1):
                for oy in (0, 1):
                    nodes.append((ix + ox) + (nx + 1) * ((iy + oy) + (ny + 1) * top))
    return np.unique(np.asarray(nodes, dtype=np.int64))


def bracket(shape=(256, 128, 128), seed=0, sigma=4.0, vsize=1e-3, material=ALUMINUM,
            load_n=5000.0, patch=16):
    """Seeded noise part: z=0 face nodes of solid voxels clamped on XYZ,
    ``load_n`` in -z on the top-surface nodes under a centred patch."""
    nx, ny, nz = shape
    E, nu = material
    solid = noise_solid(shape, seed, sigma)
    ex, ey = np.nonzero(solid[:, :, 0])
    base_nodes = _node_ids_of_elements(ex, ey, np.zeros_like(ex), nx, ny)[:, :4]
    load_nodes = _top_patch_nodes(solid, nx // 2, ny // 2, patch // 2, patch // 2)
    n_nodes = (nx + 1) * (ny + 1) * (nz + 1)
    f = np.zeros(3 * n_nodes)
    if load_nodes.size:
        f[3 * load_nodes + 2] = -load_n / load_nodes.size
    nelem = nx * ny * nz
    active = solid.ravel()
    return {
        "name": f"bracket_{nx}x{ny}x{nz}_s{seed}", "dims": shape, "vsize": vsize,
        "seed": seed, "active": active,
        "E_stiff": np.full(nelem, E * vsize), "E_stress": np.full(nelem, E),
        "nu": nu, "fixed_dofs": _dofs_of_nodes(base_nodes.ravel()), "f": f,
    }


def two_material_part(shape=(512, 256, 256), seed=0, sigma=4.0, vsize=1e-3,
                      mat_a=STEEL, mat_b=ABS, load_n=5000.0, patch=16):
    """Noise part whose voxels are split between two materials by a second,
    independent blurred-noise threshold (per-voxel E and nu)."""
    prob = bracket(shape, seed, sigma, vsize, mat_a, load_n, patch)
    rng = np.random.default_rng(seed + 7919)
    second = _blurred_noise(rng, shape, sigma)
    is_a = (second > np.median(second)).ravel()
    E = np.where(is_a, mat_a[0], mat_b[0])
    prob.update(name=f"twomat_{shape[0]}x{shape[1]}x{shape[2]}_s{seed}",
                E_stiff=E * vsize, E_stress=E.astype(float),
                nu=np.where(is_a, mat_a[1], mat_b[1]).astype(float))
    return prob


def drop_unsupported(prob):
    """The island step every job of the reference passes through before its
    solve (``core/solve_worker.py:274-287`` calling ``fea.drop_unsupported_islands``,
    ``core/fea.py:164-227``): keep only the active voxels joined to a support
    by a chain of face-adjacent active voxels, seeded by every voxel that
    touches a fixed node.  Material hanging on by an edge or a corner (the
    26-connected labelling of ``noise_solid`` keeps it) is a hinge whose
    rigid rotation only the e_min voids resist; this drops it.  The loads and
    supports are left as they are, as in the reference.  Returns a new dict
    with ``active`` restricted and ``islands_removed`` = voxels dropped."""
    from scipy import ndimage
    nx, ny, nz = prob["dims"]
    active = prob["active"].reshape(nx, ny, nz)
    fixed_nodes = np.unique(np.asarray(prob["fixed_dofs"], dtype=np.int64) // 3)
    node_fixed = np.zeros((nx + 1) * (ny + 1) * (nz + 1), dtype=bool)
    node_fixed[fixed_nodes] = True
    node_fixed = node_fixed.reshape(nz + 1, ny + 1, nx + 1).transpose(2, 1, 0)
    seed = np.zeros((nx, ny, nz), dtype=bool)
    for ox in (0, 1):
        for oy in (0, 1):
            for oz in (0, 1):
                seed |= node_fixed[ox:ox + nx, oy:oy + ny, oz:oz + nz]
    lab, _ = ndimage.label(active)          # default structure: 6-connected
    keep_labels = np.unique(lab[seed & active])
    keep_labels = keep_labels[keep_labels > 0]
    out = dict(prob)
    if keep_labels.size == 0:
        out["islands_removed"] = 0
        return out
    kept = np.isin(lab, keep_labels)
    out["active"] = kept.ravel()
    out["islands_removed"] = int(active.sum() - kept.sum())
    return out


def load_cases(prob, k, seed, patch=8, mag=(1e3, 1e4)):
    """(k, ndof) block of right-hand sides on one geometry: unit direction
    uniform on the sphere, magnitude uniform in ``mag``, each on a random
    ``patch`` x ``patch`` top patch."""
    nx, ny, nz = prob["dims"]
    solid = prob["active"].reshape(nx, ny, nz)
    rng = np.random.default_rng(seed)
    F = np.zeros((k, 3 * (nx + 1) * (ny + 1) * (nz + 1)))
    for i in range(k):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        m = rng.uniform(*mag)
        for _ in range(64):
            cx = int(rng.integers(patch // 2, max(nx - patch // 2, patch // 2 + 1)))
            cy = int(rng.integers(patch // 2, max(ny - patch // 2, patch // 2 + 1)))
            nodes = _top_patch_nodes(solid, cx, cy, patch // 2, patch // 2)
            if nodes.size:
                break
        for c in range(3):
            F[i, 3 * nodes + c] = d[c] * m / nodes.size
    return F
