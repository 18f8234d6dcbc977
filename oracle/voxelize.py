"""CPU restatement of the reference's point-in-mesh inside test (test
infrastructure: the oracle of the device voxelization kernel).

Follows VoxelSim-FEA core/inside_worker.py: voxel_centers / node_coords
(lines 68-89, element order iz-fastest, node order x-fastest) and
_inside_mask_numpy (lines 105-147): one fixed ray direction
(1, 0.0073301, 0.0031337) normalised, Moeller-Trumbore with the same
tolerances, odd crossing count = inside.  (The reference switches to
trimesh.contains for meshes of 600+ triangles when trimesh is installed; it is
not installed here, and the parity ray cast is the path pinned.)
"""

import numpy as np

RAY_DIR = np.array([1.0, 0.0073301, 0.0031337])
RAY_DIR = RAY_DIR / np.linalg.norm(RAY_DIR)


def voxel_centers(dims, origin, vsize):
    nx, ny, nz = dims
    o = np.asarray(origin, dtype=np.float64)
    xs = (np.arange(nx) + 0.5) * float(vsize) + o[0]
    ys = (np.arange(ny) + 0.5) * float(vsize) + o[1]
    zs = (np.arange(nz) + 0.5) * float(vsize) + o[2]
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def node_coords(dims, origin, vsize):
    nx, ny, nz = dims
    n = np.arange((nx + 1) * (ny + 1) * (nz + 1))
    ijk = np.stack([n % (nx + 1), (n // (nx + 1)) % (ny + 1), n // ((nx + 1) * (ny + 1))], axis=1)
    return ijk.astype(np.float64) * float(vsize) + np.asarray(origin, dtype=np.float64)


def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def inside_mask(verts, faces, points, direction=None, chunk=4096):
    """bool (len(points),): odd number of forward crossings of the ray."""
    d = RAY_DIR if direction is None else np.asarray(direction, dtype=np.float64)
    V = np.asarray(verts, dtype=np.float64)
    F = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    P = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(len(P), dtype=bool)
    if len(P) == 0 or len(F) == 0:
        return out
    v0, v1, v2 = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    e1, e2 = v1 - v0, v2 - v0
    pv = _cross(np.broadcast_to(d, e2.shape), e2)
    det = _dot(e1, pv)
    par = np.abs(det) < 1e-9
    inv = np.zeros_like(det)
    inv[~par] = 1.0 / det[~par]
    for s in range(0, len(P), chunk):
        p = P[s:s + chunk]
        tv = p[:, None, :] - v0[None, :, :]
        u = _dot(tv, pv[None]) * inv[None]
        q = _cross(tv, np.broadcast_to(e1[None], tv.shape))
        v = _dot(np.broadcast_to(d, q.shape), q) * inv[None]
        t = _dot(np.broadcast_to(e2[None], q.shape), q) * inv[None]
        hit = ~par[None] & (u >= -1e-7) & (v >= -1e-7) & (u + v <= 1.0 + 1e-7) & (t > 1e-7)
        out[s:s + chunk] = (hit.sum(axis=1) % 2) == 1
    return out
