"""Point-in-mesh inside test (voxelization) on the device -- the drop-in for
VoxelSim-FEA core/inside_worker.py (voxel_centers, node_coords, inside_mask).

The test is the reference's fixed-direction parity ray cast
(_inside_mask_numpy, inside_worker.py:105-147) computed by libvoxfea's
``vf_inside_*`` kernels with the reference's arithmetic, operation for
operation in FP64, so the masks are the reference's bit for bit.  The
reference's optional trimesh broad-phase (used when trimesh is installed and
the mesh has 600+ triangles) is a different algorithm; the ray cast is used
for every mesh size here.  There is no CPU fallback: the library is required.
"""

import ctypes

import numpy as np

from . import _lib

RAY_DIR = np.array([1.0, 0.0073301, 0.0031337])
RAY_DIR = RAY_DIR / np.linalg.norm(RAY_DIR)      # inside_worker.py:48-49


def voxel_centers(dims, origin, vsize):
    """(nelem, 3) voxel centers, element order iz-fastest (inside_worker.py:68-76)."""
    nx, ny, nz = dims
    o = np.asarray(origin, dtype=np.float64)
    xs = (np.arange(nx) + 0.5) * float(vsize) + o[0]
    ys = (np.arange(ny) + 0.5) * float(vsize) + o[1]
    zs = (np.arange(nz) + 0.5) * float(vsize) + o[2]
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def node_coords(dims, origin, vsize):
    """(nnodes, 3) grid nodes, node order x-fastest (inside_worker.py:79-89)."""
    nx, ny, nz = dims
    n = np.arange((nx + 1) * (ny + 1) * (nz + 1))
    ijk = np.stack([n % (nx + 1), (n // (nx + 1)) % (ny + 1), n // ((nx + 1) * (ny + 1))], axis=1)
    return ijk.astype(np.float64) * float(vsize) + np.asarray(origin, dtype=np.float64)


def _mesh(verts, faces):
    V = np.ascontiguousarray(np.asarray(verts, dtype=np.float64).reshape(-1, 3))
    F = np.ascontiguousarray(np.asarray(faces, dtype=np.int64).reshape(-1, 3))
    return V, F


def _dir(direction):
    d = RAY_DIR if direction is None else np.asarray(direction, dtype=np.float64)
    return np.ascontiguousarray(d, dtype=np.float64)


def inside_mask(verts, faces, points, direction=None, prefer_trimesh=True, progress_cb=None):
    """bool (len(points),) inside mask (inside_worker.py:inside_mask)."""
    del prefer_trimesh
    V, F = _mesh(verts, faces)
    P = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
    out = np.zeros(len(P), dtype=np.uint8)
    d = _dir(direction)
    rc = _lib.load().vf_inside_points(_lib.ptr(V), len(V), F.ctypes.data_as(ctypes.c_void_p), len(F),
                                      _lib.ptr(P), len(P), _lib.ptr(d), out.ctypes.data_as(ctypes.c_void_p))
    _lib.check(rc, None, "inside_mask")
    if progress_cb is not None:
        progress_cb(len(P))
    return out.astype(bool)


def inside_grid(verts, faces, dims, origin, vsize, target="centers", direction=None):
    """Inside mask of the voxel centers (target "centers") or the grid nodes
    ("nodes") of a grid, the points generated on the device."""
    V, F = _mesh(verts, faces)
    dims3 = (ctypes.c_int32 * 3)(*[int(v) for v in dims])
    o = np.ascontiguousarray(np.asarray(origin, dtype=np.float64))
    nx, ny, nz = (int(v) for v in dims)
    n = nx * ny * nz if target == "centers" else (nx + 1) * (ny + 1) * (nz + 1)
    out = np.zeros(n, dtype=np.uint8)
    d = _dir(direction)
    rc = _lib.load().vf_inside_grid(_lib.ptr(V), len(V), F.ctypes.data_as(ctypes.c_void_p), len(F), dims3,
                                    _lib.ptr(o), float(vsize), 0 if target == "centers" else 1, _lib.ptr(d),
                                    out.ctypes.data_as(ctypes.c_void_p))
    _lib.check(rc, None, "inside_grid")
    return out.astype(bool)
