"""VoxelFEA facade (oracle, test-only).

Restates VoxelSim-FEA ``core/fea.py:234-626`` on the CPU:

* active-DOF compression (fea.py:266-279)
* ``set_fixed`` (fea.py:357-369)
* ``_apply_K`` / ``_diagonal`` (fea.py:374-398)
* ``solve`` dispatch: MG with e_min voids (fea.py:400-495), falling back to
  Jacobi-PCG (fea.py:497-593) when the MG stall guard fires
* ``element_strain_energy`` (fea.py:595-602)
* ``element_von_mises_stress`` (fea.py:604-626)
"""

import numpy as np

from .hex8 import build_edof, hex8_b_c, hex8_ke
from .mg import MGOracle, StallError


class VoxelFEAOracle:
    def __init__(self, nx, ny, nz, nu=0.3, e_min=1e-9, active_elems=None,
                 use_multigrid=True, max_levels=6):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nelem = nx * ny * nz
        self.ndof_full = 3 * (nx + 1) * (ny + 1) * (nz + 1)
        self.e_min = e_min
        self.nu = nu
        self.use_multigrid = use_multigrid
        self.max_levels = max_levels
        self.KE = hex8_ke(1.0, nu)
        self._B0, self._C0 = hex8_b_c(nu)
        self.edof_full = build_edof(nx, ny, nz)
        if active_elems is None:
            self.active_elems = np.ones(self.nelem, dtype=bool)
        else:
            self.active_elems = np.asarray(active_elems, dtype=bool).ravel()
        edof_a = self.edof_full[self.active_elems]
        used = np.unique(edof_a)
        remap = -np.ones(self.ndof_full, dtype=np.int64)
        remap[used] = np.arange(used.size)
        self.used_dofs = used
        self.remap = remap
        self.ndof = int(used.size)
        self.edof = remap[edof_a]
        self.free = None
        self._fixed_dofs_full = np.zeros(0, dtype=np.int64)
        self.last_iters = 0
        self.last_converged = None
        self.last_resid_ratio = float("nan")
        self.resid_history = []
        self.solved_with = None

    def set_fixed(self, fixed_dofs):
        fixed_dofs = np.asarray(fixed_dofs, dtype=np.int64)
        self._fixed_dofs_full = fixed_dofs
        free = np.ones(self.ndof, dtype=bool)
        fd = self.remap[fixed_dofs]
        free[fd[fd >= 0]] = False
        self.free = free

    def _apply_K(self, u, Evec_a):
        ue = u[self.edof]
        ke_ue = (ue @ self.KE.T) * Evec_a[:, None]
        return np.bincount(self.edof.ravel(), weights=ke_ue.ravel(), minlength=self.ndof)

    def _diagonal(self, Evec_a):
        contrib = Evec_a[:, None] * np.diag(self.KE)[None, :]
        d = np.bincount(self.edof.ravel(), weights=contrib.ravel(), minlength=self.ndof)
        return np.where(d == 0, 1.0, d)

    def solve(self, Evec, f, tol=1e-4, max_cg=None, x0=None, progress_cb=None):
        if self.free is None:
            raise RuntimeError("call set_fixed() before solve()")
        if self.use_multigrid:
            mg = MGOracle(self.nx, self.ny, self.nz, self._fixed_dofs_full, nu=self.nu,
                          max_levels=self.max_levels)
            E_full = np.asarray(Evec, dtype=float)
            E_mg = np.where(self.active_elems, E_full, E_full * self.e_min)
            try:
                u = mg.solve(E_mg, np.asarray(f, dtype=float), tol=tol, max_cg=max_cg,
                             x0=x0, progress_cb=progress_cb)
                self.last_iters = mg.last_iters
                self.last_converged = mg.last_converged
                self.last_resid_ratio = mg.last_resid_ratio
                self.resid_history = list(mg.resid_history)
                self.solved_with = "multigrid"
                return u
            except StallError:
                self.use_multigrid = False
        self.solved_with = "jacobi"
        return self.solve_jacobi(Evec, f, tol=tol, max_cg=max_cg, x0=x0,
                                 progress_cb=progress_cb)

    def solve_jacobi(self, Evec, f, tol=1e-4, max_cg=None, x0=None, progress_cb=None):
        """Active-restricted Jacobi-PCG (fea.py:497-593)."""
        free = self.free
        Evec_a = np.asarray(Evec, dtype=float)[self.active_elems]
        f_r = np.asarray(f, dtype=float)[self.used_dofs]
        Minv = 1.0 / self._diagonal(Evec_a)
        self.last_iters = 0
        self.last_converged = False
        self.last_resid_ratio = float("nan")
        self.resid_history = []
        if x0 is None:
            u = np.zeros(self.ndof)
            r = f_r.copy()
        else:
            u = np.where(free, np.asarray(x0, dtype=float)[self.used_dofs], 0.0)
            r = f_r - self._apply_K(u, Evec_a)
        r = np.where(free, r, 0.0)
        z = np.where(free, Minv * r, 0.0)
        p = z.copy()
        rz = float(r @ z)
        fnorm = float(np.linalg.norm(np.where(free, f_r, 0.0)))
        if fnorm == 0:
            self.last_converged = True
            return np.zeros(self.ndof_full)
        max_cg = max_cg or 4 * int(free.sum())
        for it in range(max_cg):
            Kp = np.where(free, self._apply_K(p, Evec_a), 0.0)
            pKp = float(p @ Kp)
            if pKp == 0.0:
                self.last_converged = self.last_resid_ratio < tol
                break
            alpha = rz / pKp
            u = u + alpha * p
            r = r - alpha * Kp
            self.last_iters = it + 1
            self.last_resid_ratio = float(np.linalg.norm(np.where(free, r, 0.0))) / fnorm
            self.resid_history.append(self.last_resid_ratio)
            if progress_cb is not None:
                progress_cb(self.last_iters, self.last_resid_ratio, tol)
            if self.last_resid_ratio < tol:
                self.last_converged = True
                break
            z = np.where(free, Minv * r, 0.0)
            rz_new = float(r @ z)
            p = z.copy() if rz == 0.0 else z + (rz_new / rz) * p
            p = np.where(free, p, 0.0)
            rz = rz_new
        u = np.where(free, u, 0.0)
        u_full = np.zeros(self.ndof_full)
        u_full[self.used_dofs] = u
        return u_full

    def element_strain_energy(self, u_full):
        u = np.asarray(u_full)
        ce = np.zeros(self.nelem)
        ue = u[self.edof_full[self.active_elems]]
        ce[self.active_elems] = np.einsum("ei,ei->e", ue, ue @ self.KE.T)
        return ce

    def element_von_mises_stress(self, u_full, Evec):
        u = np.asarray(u_full)
        vm = np.zeros(self.nelem)
        if not np.any(self.active_elems):
            return vm
        ue = u[self.edof_full[self.active_elems]]
        stress = (ue @ self._B0.T) @ self._C0.T
        stress = stress * np.asarray(Evec, dtype=float)[self.active_elems][:, None]
        sx, sy, sz = stress[:, 0], stress[:, 1], stress[:, 2]
        txy, tyz, tzx = stress[:, 3], stress[:, 4], stress[:, 5]
        vm[self.active_elems] = np.sqrt(np.maximum(
            0.5 * ((sx - sy) ** 2 + (sy - sz) ** 2 + (sz - sx) ** 2)
            + 3.0 * (txy ** 2 + tyz ** 2 + tzx ** 2), 0.0))
        return vm


def true_residual(nx, ny, nz, E_full, fixed_dofs, f, u, active=None, e_min=1e-9, nu=0.3):
    """||mask(f - K u)|| / ||mask(f)|| with the full-grid FP64 operator.

    ``active`` given: inactive elements carry e_min*E (the MG convention,
    fea.py:467-469)."""
    E = np.asarray(E_full, dtype=float)
    if active is not None:
        E = np.where(np.asarray(active, bool).ravel(), E, E * e_min)
    edof = build_edof(nx, ny, nz)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    KE = hex8_ke(1.0, nu)
    free = np.ones(ndof, dtype=bool)
    free[np.asarray(fixed_dofs, dtype=np.int64)] = False
    fm = np.where(free, f, 0.0)
    um = np.where(free, u, 0.0)
    Ku = np.bincount(edof.ravel(), weights=((um[edof] @ KE.T) * E[:, None]).ravel(),
                     minlength=ndof)
    r = np.where(free, fm - Ku, 0.0)
    return float(np.linalg.norm(r) / np.linalg.norm(fm))
