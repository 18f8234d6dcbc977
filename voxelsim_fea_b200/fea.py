"""Linear-elastic voxel FEA facade on the B200 -- drop-in for VoxelSim-FEA's
``core/fea.py`` (``VoxelFEA``, ``build_edof``, ``_hex8_KE``, ``_hex8_B_C``,
``drop_unsupported_islands``).

``VoxelFEA`` keeps the reference's constructor, ``set_fixed`` / ``solve`` /
``element_von_mises_stress`` / ``element_strain_energy`` / ``close`` contract and
its public attributes (core/fea.py:234-626).  ``solve`` runs the multigrid
solver with e_min voids on the full grid (fea.py:438-495) and falls back to
Jacobi-PCG restricted to the active elements (fea.py:497-593) if the multigrid
solve raises -- both on the device.  The multigrid default here is the
robust B200 hierarchy (Galerkin coarse operators, direct coarsest solve):
the reference's rediscretized hierarchy does not converge on noise geometry.
"""

import ctypes

import numpy as np

from . import _lib, compute_plan
from .multigrid import MGSolver, SolverOptions


def _hex8_tables(nu):
    KE = np.empty(576)
    KL = np.empty(576)
    KM = np.empty(576)
    B0 = np.empty(144)
    _lib.check(_lib.load().vf_hex8_tables(float(nu), _lib.ptr(KE), _lib.ptr(KL), _lib.ptr(KM),
                                          _lib.ptr(B0)))
    return KE.reshape(24, 24), KL.reshape(24, 24), KM.reshape(24, 24), B0.reshape(6, 24)


def _hex8_KE(E=1.0, nu=0.3):
    """24x24 unit-cube stiffness (core/fea.py:31-76), from libvoxfea's tables."""
    return E * _hex8_tables(nu)[0]


def _hex8_B_C(nu=0.3):
    """Centroid B (6x24) and unit-E C (6x6) (core/fea.py:79-122)."""
    B0 = _hex8_tables(nu)[3]
    c = 1.0 / ((1 + nu) * (1 - 2 * nu))
    g = (1 - 2 * nu) / 2
    C = c * np.array([[1 - nu, nu, nu, 0, 0, 0], [nu, 1 - nu, nu, 0, 0, 0],
                      [nu, nu, 1 - nu, 0, 0, 0], [0, 0, 0, g, 0, 0],
                      [0, 0, 0, 0, g, 0], [0, 0, 0, 0, 0, g]])
    return B0, C


def _node_id(ix, iy, iz, nx, ny):
    return ix + (nx + 1) * (iy + (ny + 1) * iz)


def build_edof(nx, ny, nz):
    """(nelem, 24) global DOF ids, iz-fastest element order (core/fea.py:133-148)."""
    ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    offs = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    edof = np.empty((ex.size, 24), dtype=np.int64)
    for k, (ox, oy, oz) in enumerate(offs):
        nid = _node_id(ex + ox, ey + oy, ez + oz, nx, ny)
        for c in range(3):
            edof[:, 3 * k + c] = 3 * nid + c
    return edof


def drop_unsupported_islands(active3d, fixed_dofs):
    """Keep only active voxels 6-connected to a voxel touching a fixed node
    (core/fea.py:207-227); device flood fill.  Returns (kept3d, n_removed)."""
    active3d = np.asarray(active3d, dtype=bool)
    nx, ny, nz = active3d.shape
    act = np.ascontiguousarray(active3d.ravel().astype(np.uint8))
    fd = np.ascontiguousarray(np.asarray(fixed_dofs, dtype=np.int64).ravel())
    kept = np.empty_like(act)
    nrem = ctypes.c_int64()
    _lib.check(_lib.load().vf_drop_unsupported_islands(nx, ny, nz, _lib.ptr(act), _lib.ptr(fd), fd.size,
                                                       _lib.ptr(kept), ctypes.byref(nrem)),
               None, "drop_unsupported_islands")
    return kept.astype(bool).reshape(nx, ny, nz), int(nrem.value)


class VoxelFEA:
    """Solves K(E) u = f matrix-free over the active elements, on the B200."""

    def __init__(self, nx, ny, nz, nu=0.3, e_min=1e-9, active_elems=None, compute_mode="AUTO",
                 cpu_threads=0, verbose=False, use_multigrid=True, mg_options=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nelem = nx * ny * nz
        self.ndof_full = 3 * (nx + 1) * (ny + 1) * (nz + 1)
        self.e_min = e_min
        self.nu = nu
        self._compute_mode = compute_mode
        self._cpu_threads = cpu_threads
        self.use_multigrid = use_multigrid
        self.mg_options = mg_options if mg_options is not None else SolverOptions.robust()
        self._mg = None
        self._jac = None
        self._fixed_dofs_full = np.zeros(0, dtype=np.int64)
        self.KE, _, _, B0 = _hex8_tables(nu)
        self._B0, self._C0 = _hex8_B_C(nu)
        if active_elems is None:
            self.active_elems = np.ones(self.nelem, dtype=bool)
        else:
            self.active_elems = np.asarray(active_elems, dtype=bool).ravel()
        # active-DOF compression (fea.py:271-279): node-level bookkeeping only
        used_nodes = self._used_nodes()
        used = np.sort(np.concatenate([3 * used_nodes + c for c in range(3)]))
        remap = -np.ones(self.ndof_full, dtype=np.int64)
        remap[used] = np.arange(used.size)
        self.used_dofs = used
        self.remap = remap
        self.ndof = int(used.size)
        self.free = None
        self._diag = None
        self.verbose = verbose
        self.last_iters = 0
        self.last_converged = None
        self.last_resid_ratio = float("nan")
        self.resid_history = []
        self.plan = compute_plan.choose(self.ndof, mode=compute_mode, cpu_threads=cpu_threads,
                                        verbose=verbose)
        self._edof_full = None

    def _used_nodes(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        a = self.active_elems.reshape(nx, ny, nz)
        used = np.zeros((nx + 1, ny + 1, nz + 1), dtype=bool)
        for ox in (0, 1):
            for oy in (0, 1):
                for oz in (0, 1):
                    used[ox:ox + nx, oy:oy + ny, oz:oz + nz] |= a
        ix, iy, iz = np.nonzero(used)
        return np.sort(_node_id(ix, iy, iz, nx, ny))

    @property
    def edof_full(self):
        """(nelem, 24) connectivity (fea.py:264), built on first access."""
        if self._edof_full is None:
            self._edof_full = build_edof(self.nx, self.ny, self.nz)
        return self._edof_full

    @property
    def edof(self):
        """Reduced connectivity of the active elements (fea.py:279)."""
        return self.remap[self.edof_full[self.active_elems]]

    def close(self):
        for attr in ("_mg", "_jac"):
            obj = getattr(self, attr)
            if obj is not None:
                try:
                    obj.close()
                except Exception:
                    pass
                setattr(self, attr, None)

    def set_fixed(self, fixed_dofs):
        """fixed_dofs: original global DOF ids to constrain (fea.py:357-369)."""
        fixed_dofs = np.asarray(fixed_dofs, dtype=np.int64)
        self._fixed_dofs_full = fixed_dofs
        free = np.ones(self.ndof, dtype=bool)
        fd = self.remap[fixed_dofs]
        free[fd[fd >= 0]] = False
        self.free = free
        for obj in (self._mg, self._jac):
            if obj is not None:
                obj._build_free(fixed_dofs)

    def solve(self, Evec, f, tol=1e-4, max_cg=None, x0=None, progress_cb=None, nu_elem=None):
        """Preconditioned CG; returns the full-length u (fea.py:400-436)."""
        if self.free is None:
            raise RuntimeError("call set_fixed() before solve()")
        if self.use_multigrid:
            u = self._solve_multigrid(Evec, f, tol, max_cg, x0, progress_cb, nu_elem)
            if u is not None:
                return u
        return self._solve_jacobi(Evec, f, tol=tol, max_cg=max_cg, x0=x0, progress_cb=progress_cb,
                                  nu_elem=nu_elem)

    def _solve_multigrid(self, Evec, f, tol, max_cg, x0, progress_cb, nu_elem=None):
        if self._mg is None:
            try:
                self._mg = MGSolver(self.nx, self.ny, self.nz, self._fixed_dofs_full, nu=self.nu,
                                    compute_mode=self._compute_mode, cpu_threads=self._cpu_threads,
                                    verbose=self.verbose, options=self.mg_options)
            except Exception as exc:
                print(f"[VoxelSim FEA] MGSolver construction failed for {self.nx}x{self.ny}x{self.nz} "
                      f"(mode={self._compute_mode}): {exc}\n[VoxelSim FEA] Falling back to plain "
                      f"Jacobi-PCG (no multigrid preconditioning) for this solve.")
                self.use_multigrid = False
                self._mg = None
                return None
        E_full = np.asarray(Evec, dtype=float)
        E_mg = np.where(self.active_elems, E_full, E_full * self.e_min)   # fea.py:467-469
        try:
            u = self._mg.solve(E_mg, np.asarray(f, dtype=float), tol=tol, max_cg=max_cg, x0=x0,
                               progress_cb=progress_cb, nu_elem=nu_elem)
        except Exception as exc:
            print(f"[VoxelSim FEA] MGSolver.solve() failed for {self.nx}x{self.ny}x{self.nz}: {exc}\n"
                  f"[VoxelSim FEA] Falling back to plain Jacobi-PCG (no multigrid preconditioning) "
                  f"for this solve.")
            self.use_multigrid = False
            self._mg.close()
            self._mg = None
            return None
        self.last_iters = self._mg.last_iters
        self.last_converged = self._mg.last_converged
        self.last_resid_ratio = self._mg.last_resid_ratio
        self.resid_history = list(self._mg.resid_history)
        return u

    def _solve_jacobi(self, Evec, f, tol=1e-4, max_cg=None, x0=None, progress_cb=None, nu_elem=None):
        """Jacobi-PCG on the active elements' DOFs (fea.py:497-593), on the device."""
        if self.free is None:
            raise RuntimeError("call set_fixed() before solve()")
        if self._jac is None:
            opts = SolverOptions(precision="fp64", device=self.mg_options.device,
                                 check_every=self.mg_options.check_every)
            self._jac = MGSolver(self.nx, self.ny, self.nz, self._fixed_dofs_full, nu=self.nu,
                                 compute_mode=self._compute_mode, verbose=self.verbose, options=opts,
                                 method=_lib.VF_METHOD_JACOBI)
            act = np.ascontiguousarray(self.active_elems.astype(np.uint8))
            _lib.check(_lib.load().vf_set_active(self._jac._handle(), _lib.ptr(act)), self._jac._h)
        max_cg = max_cg or 4 * int(self.free.sum())
        self.last_iters = 0
        self.last_converged = False
        self.last_resid_ratio = float("nan")
        self.resid_history = []
        u = self._jac.solve(Evec, f, tol=tol, max_cg=max_cg, x0=x0, progress_cb=progress_cb,
                            nu_elem=nu_elem)
        if self._jac.last_info is not None and self._jac.last_info.iters < 0:
            self.last_converged = True            # zero load (fea.py:543-545)
            return u
        self.last_iters = self._jac.last_iters
        self.last_converged = bool(self._jac.last_converged)
        self.last_resid_ratio = self._jac.last_resid_ratio
        self.resid_history = list(self._jac.resid_history)
        return u

    def element_strain_energy(self, u_full):
        """Per-element u_e^T KE u_e (fea.py:595-602), zeros outside the active set."""
        h = self._any_handle()
        u = _lib.f64(np.asarray(u_full, dtype=float).ravel())
        act = np.ascontiguousarray(self.active_elems.astype(np.uint8))
        out = np.empty(self.nelem)
        _lib.check(_lib.load().vf_strain_energy(h._handle(), _lib.ptr(u), _lib.ptr(act), _lib.ptr(out)),
                   h._h)
        return out

    def element_von_mises_stress(self, u_full, Evec, nu_elem=None):
        """Per-element centroid von Mises stress (fea.py:604-626)."""
        h = self._any_handle()
        u = _lib.f64(np.asarray(u_full, dtype=float).ravel())
        E = _lib.f64(np.asarray(Evec, dtype=float).ravel())
        nu_e = None if nu_elem is None else _lib.f64(np.asarray(nu_elem, dtype=float).ravel())
        act = np.ascontiguousarray(self.active_elems.astype(np.uint8))
        out = np.empty(self.nelem)
        _lib.check(_lib.load().vf_von_mises(h._handle(), _lib.ptr(u), _lib.ptr(E), _lib.ptr(nu_e),
                                            _lib.ptr(act), _lib.ptr(out)), h._h)
        return out

    def _any_handle(self):
        for obj in (self._mg, self._jac):
            if obj is not None and obj._h is not None:
                return obj
        # post-processing without a prior solve: a single-level handle
        self._jac = MGSolver(self.nx, self.ny, self.nz, self._fixed_dofs_full, nu=self.nu,
                             compute_mode=self._compute_mode, options=SolverOptions(),
                             method=_lib.VF_METHOD_JACOBI)
        return self._jac
