"""Sparse Galerkin coarse operators (oracle, test-only).

Not a reference algorithm: the reference rediscretizes its coarse levels
(core/multigrid.py:281-315).  The CUDA path can instead build

    A_{l+1} = D_{l+1} P^T D_l A_l D_l P D_{l+1}

with the reference's trilinear P (``mg.prolong_op``, multigrid.py:42-73),
D_0 the Dirichlet mask and D_{l+1} the DOFs whose Galerkin diagonal is
non-zero.  This module assembles the same operators with scipy.sparse so the
device stencils can be checked entry by entry (through their action).
"""

import numpy as np
import scipy.sparse as sp

from .hex8 import build_edof, hex8_ke, lame_split
from .mg import level_dims, node_dims, prolong_op


def fine_matrix(nx, ny, nz, E, nu=0.3, lam=None, mu=None):
    """Assembled K = sum_e E_e Ke (or lam_e K_lam + mu_e K_mu) as CSR."""
    edof = build_edof(nx, ny, nz)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    if lam is None:
        KE = hex8_ke(1.0, nu)
        vals = (np.asarray(E, float)[:, None, None] * KE[None]).ravel()
    else:
        KL, KM = lame_split()
        vals = (np.asarray(lam, float)[:, None, None] * KL[None]
                + np.asarray(mu, float)[:, None, None] * KM[None]).ravel()
    rows = np.repeat(edof, 24, axis=1).ravel()
    cols = np.tile(edof, (1, 24)).ravel()
    return sp.csr_matrix((vals, (rows, cols)), shape=(ndof, ndof))


def prolong_matrix(fine_dims_el, coarse_dims_el):
    """(3 Nf) x (3 Nc) trilinear P acting on interleaved DOFs."""
    idx, w = prolong_op(node_dims(*fine_dims_el), node_dims(*coarse_dims_el))
    Nf = idx.shape[0]
    Nc = int(np.prod(node_dims(*coarse_dims_el)))
    rows, cols, vals = [], [], []
    for c in range(3):
        rows.append(np.repeat(3 * np.arange(Nf) + c, 8))
        cols.append((3 * idx + c).ravel())
        vals.append(w.ravel())
    P = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(3 * Nf, 3 * Nc))
    P.sum_duplicates()
    return P


def galerkin_hierarchy(nx, ny, nz, E, fixed_dofs, nu=0.3, min_elems=4, max_levels=6,
                       lam=None, mu=None):
    """[(A_l, free_l)] for every level; A_0 is the masked fine operator."""
    dims = level_dims(nx, ny, nz, min_elems, max_levels)
    K = fine_matrix(nx, ny, nz, E, nu, lam, mu)
    free = np.ones(K.shape[0], dtype=bool)
    free[np.asarray(fixed_dofs, dtype=np.int64)] = False
    D = sp.diags(free.astype(float))
    A = (D @ K @ D).tocsr()
    out = [(A, free)]
    for li in range(1, len(dims)):
        P = prolong_matrix(dims[li - 1], dims[li])
        Dp = sp.diags(out[-1][1].astype(float))
        Ac = (P.T @ Dp @ out[-1][0] @ Dp @ P).tocsr()
        fc = Ac.diagonal() > 0
        Dc = sp.diags(fc.astype(float))
        out.append(((Dc @ Ac @ Dc).tocsr(), fc))
    return out


def _lambda_max(A, dinv, free, iters=30, seed=0):
    """Power-iteration estimate of lambda_max(D^-1 A) on the free DOFs."""
    x = np.random.default_rng(seed).standard_normal(A.shape[0]) * free
    lam = 0.0
    for _ in range(iters):
        y = dinv * (A @ x)
        lam = np.linalg.norm(y) / np.linalg.norm(x)
        x = y / np.linalg.norm(y)
    return lam


def smoothed_hierarchy(nx, ny, nz, E, fixed_dofs, nu=0.3, min_elems=4, max_levels=6, lam=None, mu=None,
                       omega=4.0 / 3.0, pad=1.1, smoothed=None, lams=None):
    """[(A_l, free_l)], [P_l]: Galerkin levels with smoothed prolongations.

    P_l = D_l (P - (omega / lambda_l) D_l^-1 A_l P) (one damped-Jacobi step
    applied to the trilinear P, lambda_l the padded lambda_max(D^-1 A_l)),
    A_{l+1} = D_{l+1} P_l^T A_l P_l D_{l+1}; the coarse stencils reach two
    nodes out (125 blocks) instead of one.  Not a reference algorithm: the
    coarse space of the device hierarchy's smoothed transfers
    (vf_options.smoothed_transfers), checked against this.

    smoothed: the transfers l -> l+1 to smooth (None: all; the others use the
    trilinear P = D_l P); lams: {l: padded lambda_l} to use instead of this
    module's own power-iteration estimate (the device's, for entrywise checks)."""
    dims = level_dims(nx, ny, nz, min_elems, max_levels)
    K = fine_matrix(nx, ny, nz, E, nu, lam, mu)
    free = np.ones(K.shape[0], dtype=bool)
    free[np.asarray(fixed_dofs, dtype=np.int64)] = False
    D = sp.diags(free.astype(float))
    out = [((D @ K @ D).tocsr(), free)]
    Ps = []
    for li in range(1, len(dims)):
        A, fr = out[-1]
        P = prolong_matrix(dims[li - 1], dims[li])
        if smoothed is None or (li - 1) in smoothed:
            d = A.diagonal()
            dinv = np.where(fr & (d > 0), 1.0 / np.where(d > 0, d, 1.0), 0.0)
            lmax = lams[li - 1] if lams and (li - 1) in lams else pad * _lambda_max(A, dinv, fr)
            Psm = (sp.diags(fr.astype(float)) @ (P - (omega / lmax) * (sp.diags(dinv) @ (A @ P)))).tocsr()
        else:
            Psm = (sp.diags(fr.astype(float)) @ P).tocsr()
        Ac = (Psm.T @ A @ Psm).tocsr()
        fc = Ac.diagonal() > 0
        Dc = sp.diags(fc.astype(float))
        Ps.append((Psm @ Dc).tocsr())
        out.append(((Dc @ Ac @ Dc).tocsr(), fc))
    return out, Ps
