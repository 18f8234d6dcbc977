"""Hex8 element matrices and structured-grid connectivity (oracle, test-only).

Restates VoxelSim-FEA ``core/fea.py:27-148``:

* ``hex8_ke``      -- ``_hex8_KE``  (fea.py:31-76): 24x24 unit-cube stiffness,
                      2x2x2 Gauss quadrature, J = 0.5 I.
* ``hex8_b_c``     -- ``_hex8_B_C`` (fea.py:79-122): centroid B (6x24) and
                      unit-E C (6x6), Voigt order [xx, yy, zz, xy, yz, zx].
* ``node_id``      -- ``_node_id``  (fea.py:129-130): x-fastest node ids.
* ``build_edof``   -- ``build_edof`` (fea.py:133-148): element order is the
                      ``meshgrid(..., indexing='ij').ravel()`` order, i.e. iz
                      fastest; local node order (0,0,0),(1,0,0),(1,1,0),(0,1,0),
                      (0,0,1),(1,0,1),(1,1,1),(0,1,1).

``lame_split`` is the project's own observation (not in the reference) that
``_hex8_KE(E, nu) == lam * K_lam + mu * K_mu`` with nu-independent K_lam, K_mu,
used to support a per-voxel Poisson ratio.
"""

import numpy as np

# local corner offsets of an element, reference order (fea.py:33-36, 140-141)
CORNERS = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
           (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))


def _c_matrix(nu):
    c = 1.0 / ((1 + nu) * (1 - 2 * nu))
    g = (1 - 2 * nu) / 2
    return c * np.array([
        [1 - nu, nu, nu, 0, 0, 0],
        [nu, 1 - nu, nu, 0, 0, 0],
        [nu, nu, 1 - nu, 0, 0, 0],
        [0, 0, 0, g, 0, 0],
        [0, 0, 0, 0, g, 0],
        [0, 0, 0, 0, 0, g],
    ])


def _b_matrix(xi, eta, zeta):
    """Strain-displacement matrix of the unit cube at a reference point.

    Shape-function derivatives of the trilinear hex (fea.py:54-58), mapped by
    the constant Jacobian 0.5*I (fea.py:59-61) and laid out as in fea.py:62-74.
    """
    dN = np.zeros((3, 8))
    for i, (ox, oy, oz) in enumerate(CORNERS):
        a, b, c = 2 * ox - 1, 2 * oy - 1, 2 * oz - 1
        dN[0, i] = a * (1 + b * eta) * (1 + c * zeta) / 8.0
        dN[1, i] = b * (1 + a * xi) * (1 + c * zeta) / 8.0
        dN[2, i] = c * (1 + a * xi) * (1 + b * eta) / 8.0
    dNxyz = dN / 0.5
    B = np.zeros((6, 24))
    for i in range(8):
        bx, by, bz = dNxyz[:, i]
        c0 = 3 * i
        B[0, c0] = bx
        B[1, c0 + 1] = by
        B[2, c0 + 2] = bz
        B[3, c0] = by
        B[3, c0 + 1] = bx
        B[4, c0 + 1] = bz
        B[4, c0 + 2] = by
        B[5, c0] = bz
        B[5, c0 + 2] = bx
    return B


def hex8_ke(E=1.0, nu=0.3):
    """24x24 unit-cube stiffness (fea.py:31-76); detJ = 0.125, unit weights."""
    C = E * _c_matrix(nu)
    g = 1.0 / np.sqrt(3.0)
    KE = np.zeros((24, 24))
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                B = _b_matrix(xi, eta, zeta)
                KE += (B.T @ C @ B) * 0.125
    return KE


def hex8_b_c(nu=0.3):
    """Centroid B (6x24) and unit-E C (6x6) (fea.py:79-122)."""
    return _b_matrix(0.0, 0.0, 0.0), _c_matrix(nu)


def lame(E, nu):
    """Lame parameters (lambda, mu) of an isotropic material."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return lam, mu


def lame_split():
    """(K_lam, K_mu) with hex8_ke(E, nu) == lam*K_lam + mu*K_mu exactly.

    Obtained by integrating B^T C B with C = lam*(m m^T) + mu*diag(2,2,2,1,1,1)
    (m = [1,1,1,0,0,0]), the same quadrature as ``hex8_ke``.
    """
    m = np.array([1, 1, 1, 0, 0, 0], dtype=float)
    CL = np.outer(m, m)
    CM = np.diag([2.0, 2.0, 2.0, 1.0, 1.0, 1.0])
    g = 1.0 / np.sqrt(3.0)
    KL = np.zeros((24, 24))
    KM = np.zeros((24, 24))
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                B = _b_matrix(xi, eta, zeta)
                KL += (B.T @ CL @ B) * 0.125
                KM += (B.T @ CM @ B) * 0.125
    return KL, KM


def node_id(ix, iy, iz, nx, ny):
    """x-fastest node id (fea.py:129-130)."""
    return ix + (nx + 1) * (iy + (ny + 1) * iz)


def build_edof(nx, ny, nz):
    """(nelem, 24) global DOF ids per element, iz-fastest element order
    (fea.py:133-148)."""
    ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz),
                             indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    edof = np.empty((ex.size, 24), dtype=np.int64)
    for k, (ox, oy, oz) in enumerate(CORNERS):
        nid = node_id(ex + ox, ey + oy, ez + oz, nx, ny)
        edof[:, 3 * k] = 3 * nid
        edof[:, 3 * k + 1] = 3 * nid + 1
        edof[:, 3 * k + 2] = 3 * nid + 2
    return edof


def element_apply(u, E_elem, edof, KE, ndof):
    """y = sum_e E_e * KE u_e  (gather, GEMM, bincount scatter: fea.py:383-386,
    multigrid.py:334-337)."""
    ue = u[edof]
    ke = (ue @ KE.T) * E_elem[:, None]
    return np.bincount(edof.ravel(), weights=ke.ravel(), minlength=ndof)


def element_apply_lame(u, lam_elem, mu_elem, edof, ndof):
    """y = sum_e (lam_e K_lam + mu_e K_mu) u_e, for a per-voxel Poisson ratio."""
    KL, KM = lame_split()
    ue = u[edof]
    ke = (ue @ KL.T) * lam_elem[:, None] + (ue @ KM.T) * mu_elem[:, None]
    return np.bincount(edof.ravel(), weights=ke.ravel(), minlength=ndof)
