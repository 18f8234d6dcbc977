"""Geometric-multigrid PCG on the full voxel grid (oracle, test-only).

Restates VoxelSim-FEA ``core/multigrid.py`` on the CPU with numpy, without the
compute-plan / matvec-pool machinery (the oracle is always single-process FP64):

* ``prolong_op``            -- ``_prolong_op``  (multigrid.py:42-73)
* ``MGOracle.__init__``     -- ``MGSolver.__init__`` hierarchy (multigrid.py:141-171)
* ``MGOracle._build_free``  -- injection of the Dirichlet mask (multigrid.py:255-278)
* ``MGOracle.set_density``  -- 2x2x2 mean coarse E, g = 2^level, Jacobi diagonal
                               (multigrid.py:281-315)
* ``MGOracle.apply``        -- ``_apply`` (multigrid.py:318-341)
* ``MGOracle.smooth``       -- ``_smooth`` (multigrid.py:367-402, un-pooled branch)
* ``MGOracle.restrict``     -- ``_restrict`` (multigrid.py:404-416)
* ``MGOracle.prolongate``   -- ``_prolongate`` (multigrid.py:418-424)
* ``MGOracle.vcycle``       -- ``_vcycle`` (multigrid.py:426-436)
* ``MGOracle.solve``        -- ``solve`` (multigrid.py:439-583) incl. the stall
                               guard (494-531) and zero-denominator guards.
"""

import numpy as np

from .hex8 import build_edof, hex8_ke


def node_dims(nx, ny, nz):
    return (nx + 1, ny + 1, nz + 1)


def level_dims(nx, ny, nz, min_elems=4, max_levels=6):
    """Grid hierarchy: halve while every dim is even (multigrid.py:142-148)."""
    dims = [(nx, ny, nz)]
    while (len(dims) < max_levels and dims[-1][0] % 2 == 0
           and dims[-1][1] % 2 == 0 and dims[-1][2] % 2 == 0
           and min(dims[-1]) // 2 >= min_elems // 2 and min(dims[-1]) >= 2):
        cx, cy, cz = dims[-1]
        dims.append((cx // 2, cy // 2, cz // 2))
    return dims


def prolong_op(fine_dims, coarse_dims):
    """Trilinear P as (idx[Nf,8], w[Nf,8]) over coarse node ids (multigrid.py:42-73)."""
    Lfx, Lfy, Lfz = fine_dims
    Lcx, Lcy, Lcz = coarse_dims
    n = np.arange(Lfx * Lfy * Lfz)
    ix = n % Lfx
    iy = (n // Lfx) % Lfy
    iz = n // (Lfx * Lfy)
    cc = np.stack([ix, iy, iz], axis=1) / 2.0
    base = np.floor(cc).astype(np.int64)
    fr = cc - base
    idx = np.empty((n.size, 8), dtype=np.int64)
    w = np.empty((n.size, 8))
    corners = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0),
               (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    for k, (ox, oy, oz) in enumerate(corners):
        jx = np.clip(base[:, 0] + ox, 0, Lcx - 1)
        jy = np.clip(base[:, 1] + oy, 0, Lcy - 1)
        jz = np.clip(base[:, 2] + oz, 0, Lcz - 1)
        wx = fr[:, 0] if ox else (1.0 - fr[:, 0])
        wy = fr[:, 1] if oy else (1.0 - fr[:, 1])
        wz = fr[:, 2] if oz else (1.0 - fr[:, 2])
        idx[:, k] = jx + Lcx * (jy + Lcy * jz)
        w[:, k] = wx * wy * wz
    return idx, w


class StallError(RuntimeError):
    """Raised by the stall/divergence guard (multigrid.py:523-531)."""


class MGOracle:
    """FP64 MG-PCG with the reference's exact algorithm (numpy, CPU)."""

    def __init__(self, nx, ny, nz, fixed_dofs, nu=0.3, n_smooth=2, omega=0.6,
                 min_elems=4, max_levels=6):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nelem = nx * ny * nz
        self.ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
        self.n_smooth = n_smooth
        self.omega = omega
        self.KE = hex8_ke(1.0, nu)
        self.diagKE = np.diag(self.KE).copy()
        self.levels = []
        for li, (lx, ly, lz) in enumerate(level_dims(nx, ny, nz, min_elems, max_levels)):
            self.levels.append({
                "dims": (lx, ly, lz),
                "ndof": 3 * (lx + 1) * (ly + 1) * (lz + 1),
                "edof": build_edof(lx, ly, lz),
                "g": float(2 ** li),
            })
        self.prolong = [prolong_op(node_dims(*self.levels[i]["dims"]),
                                   node_dims(*self.levels[i + 1]["dims"]))
                        for i in range(len(self.levels) - 1)]
        self._build_free(fixed_dofs)
        self.last_iters = 0
        self.last_converged = None
        self.last_resid_ratio = float("nan")
        self.resid_history = []

    def _build_free(self, fixed_dofs):
        free0 = np.ones(self.levels[0]["ndof"], dtype=bool)
        fd = np.asarray(fixed_dofs, dtype=np.int64)
        if fd.size:
            free0[fd] = False
        self.levels[0]["free"] = free0
        prev_free = free0
        prev_dims = node_dims(*self.levels[0]["dims"])
        for li in range(1, len(self.levels)):
            Lcx, Lcy, Lcz = node_dims(*self.levels[li]["dims"])
            Lfx, Lfy, _ = prev_dims
            n = np.arange(Lcx * Lcy * Lcz)
            jx = n % Lcx
            jy = (n // Lcx) % Lcy
            jz = n // (Lcx * Lcy)
            fid = 2 * jx + Lfx * (2 * jy + Lfy * (2 * jz))
            free = np.ones(3 * n.size, dtype=bool)
            for c in range(3):
                free[3 * n + c] = prev_free[3 * fid + c]
            self.levels[li]["free"] = free
            prev_free = free
            prev_dims = (Lcx, Lcy, Lcz)

    def set_density(self, Evec_full):
        E = np.asarray(Evec_full, dtype=float)
        for li, lv in enumerate(self.levels):
            lx, ly, lz = lv["dims"]
            if li > 0:
                plx, ply, plz = self.levels[li - 1]["dims"]
                pe3 = self.levels[li - 1]["Evec"].reshape(plx, ply, plz)
                E = pe3.reshape(lx, 2, ly, 2, lz, 2).mean(axis=(1, 3, 5)).ravel()
            lv["Evec"] = E
            scaled = E * lv["g"]
            d = np.bincount(lv["edof"].ravel(),
                            weights=(scaled[:, None] * self.diagKE[None, :]).ravel(),
                            minlength=lv["ndof"])
            d = np.where(d == 0, 1.0, d)
            lv["Minv"] = 1.0 / d
            lv["_scaled"] = scaled

    def apply(self, li, u):
        lv = self.levels[li]
        ue = u[lv["edof"]]
        ke = (ue @ self.KE.T) * lv["_scaled"][:, None]
        Ku = np.bincount(lv["edof"].ravel(), weights=ke.ravel(), minlength=lv["ndof"])
        return np.where(lv["free"], Ku, 0.0)

    def smooth(self, li, u, b, iters):
        lv = self.levels[li]
        for _ in range(iters):
            r = b - self.apply(li, u)
            u = u + self.omega * np.where(lv["free"], lv["Minv"] * r, 0.0)
        return u

    def restrict(self, li, r_fine):
        idx, wt = self.prolong[li]
        Nc = self.levels[li + 1]["ndof"] // 3
        rf = r_fine.reshape(-1, 3)
        rc = np.zeros((Nc, 3))
        for c in range(3):
            rc[:, c] = np.bincount(idx.ravel(), weights=(wt * rf[:, c][:, None]).ravel(),
                                   minlength=Nc)
        return np.where(self.levels[li + 1]["free"], rc.reshape(-1), 0.0)

    def prolongate(self, li, e_coarse):
        idx, wt = self.prolong[li]
        ec = e_coarse.reshape(-1, 3)
        ef = (ec[idx] * wt[:, :, None]).sum(axis=1)
        return np.where(self.levels[li]["free"], ef.reshape(-1), 0.0)

    def vcycle(self, li, b):
        if li == len(self.levels) - 1:
            return self.smooth(li, np.zeros_like(b), b, 30)
        u = self.smooth(li, np.zeros_like(b), b, self.n_smooth)
        r = b - self.apply(li, u)
        rc = self.restrict(li, r)
        ec = self.vcycle(li + 1, rc)
        u = u + self.prolongate(li, ec)
        return self.smooth(li, u, b, self.n_smooth)

    def solve(self, Evec_full, f, tol=1e-4, max_cg=None, x0=None, progress_cb=None):
        self.resid_history = []
        self.set_density(Evec_full)
        free = self.levels[0]["free"]
        f = np.where(free, np.asarray(f, dtype=float), 0.0)
        if x0 is None:
            u = np.zeros(self.ndof)
            r = f.copy()
        else:
            u = np.where(free, np.asarray(x0, dtype=float), 0.0)
            r = f - self.apply(0, u)
        r = np.where(free, r, 0.0)
        fnorm = float(np.linalg.norm(f))
        if fnorm == 0.0:
            return np.zeros(self.ndof)
        z = self.vcycle(0, r)
        p = z.copy()
        rz = float(r @ z)
        max_cg = max_cg or 1000
        self.last_iters = 0
        self.last_converged = False
        self.last_resid_ratio = float("nan")
        best = float("inf")
        for it in range(max_cg):
            Ap = self.apply(0, p)
            pAp = float(p @ Ap)
            if pAp == 0.0:
                self.last_converged = self.last_resid_ratio < tol
                break
            alpha = rz / pAp
            u = u + alpha * p
            r = r - alpha * Ap
            self.last_iters = it + 1
            self.last_resid_ratio = float(np.linalg.norm(r)) / fnorm
            self.resid_history.append(self.last_resid_ratio)
            if progress_cb is not None:
                progress_cb(self.last_iters, self.last_resid_ratio, tol)
            if self.last_resid_ratio < tol:
                self.last_converged = True
                break
            best = min(best, self.last_resid_ratio)
            if self.last_iters >= 10 and self.last_resid_ratio > 5.0 * best:
                raise StallError(f"MG-PCG stalled/diverged at iter {self.last_iters}")
            z = self.vcycle(0, r)
            rz_new = float(r @ z)
            p = z.copy() if rz == 0.0 else z + (rz_new / rz) * p
            rz = rz_new
        return np.where(free, u, 0.0)
