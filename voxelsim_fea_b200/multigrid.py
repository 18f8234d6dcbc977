"""Geometric-multigrid PCG solver on the B200 -- drop-in for
VoxelSim-FEA's ``core/multigrid.py`` ``MGSolver``.

Same constructor signature, ``solve`` contract, attributes (``last_iters``,
``last_converged``, ``last_resid_ratio``, ``resid_history``, ``levels``,
``plan``) and error behaviour (stall guard raises ``RuntimeError``, always
printed non-convergence warning) as the reference (core/multigrid.py:85-583).
Every operator, smoother sweep, transfer and PCG update runs in libvoxfea on
the device; the host only supplies numpy inputs and receives numpy ``u``.

Default settings reproduce the reference algorithm exactly (FP64,
rediscretized coarse levels, injected Dirichlet masks, 30-sweep Jacobi coarse
"solve").  ``SolverOptions`` selects the B200 extensions:

* ``coarse="galerkin"``  R A P coarse operators (robust on void/solid noise
  geometry, where the rediscretized hierarchy stops converging);
* ``coarsest="cholesky"`` FP64 dense direct solve on the coarsest level;
* ``precision="mixed"`` the FP32 V-cycle (matvec, smoother, transfers) inside
  FP64 PCG (``mixed_mode="outer64"``, default: FP64 dots, A p, vector updates
  and coarsest solve), or FP32 CG with FP64 residual replacement
  (``"reliable"``) or iterative refinement (``"restart"``); ``"fp32"``: FP32
  PCG without refinement.
"""

import ctypes
import dataclasses
import time

import numpy as np

from . import _lib, compute_plan


def _preset_smoother(kw):
    """The presets smooth with Chebyshev polynomials wherever the chosen kernels
    take its step (modal fine kernel, symmetric coarse storage, auto damping)."""
    if kw.get("fine_kernel") == "gather" or kw.get("coarse_storage") == "full" or \
            kw.get("omega_mode", "auto") != "auto":
        return "jacobi"
    return "chebyshev"


def _preset_level_sweeps(kw):
    """With the level 1 -> 2 transfer smoothed, level 1 is smoothed once more by
    its smoothed restriction and prolongation: the presets give it one
    Chebyshev step before and after the coarse correction instead of two
    (bracket 256x128x128: 158 -> 162 iterations, 3.8 % less time to
    solution; held-out 192^3 two-material parts: 532 -> 560 iterations, 3 %
    less time)."""
    return 1 if _preset_transfers(kw) and kw.get("smoothed_transfers", 2) else 0


def _preset_transfers(kw):
    """The presets smooth the level 1 -> 2 prolongation (the 125-block coarse
    space) wherever the options allow it (Galerkin levels, auto damping,
    symmetric storage): about 1.4x fewer PCG iterations at the price of a
    heavier set-up and level 2."""
    if kw.get("coarse_storage") == "full" or kw.get("omega_mode", "auto") != "auto":
        return 0
    return 2


@dataclasses.dataclass
class SolverOptions:
    """B200 solver options beyond the reference's keyword arguments."""
    precision: str = "fp64"          # "fp64" | "mixed" | "fp32"
    coarse: str = "rediscretize"     # "rediscretize" (reference) | "galerkin"
    coarsest: str = "jacobi"         # "jacobi" (reference, 30 sweeps) | "cholesky"
    coarse_sweeps: int = 30
    stall_guard: bool = True
    check_every: int = 8             # PCG iterations per device graph launch
    use_graphs: bool = True
    device: int = 0
    inner_tol: float = 1e-2          # mixed: residual reduction between FP64 corrections
    max_outer: int = 20              # mixed: cap on FP64 corrections
    # mixed: "outer64" (FP64 PCG, FP32 V-cycle) | "reliable" (FP32 CG, residual
    # replacement) | "restart" (refinement)
    mixed_mode: str = "outer64"
    flexible: bool = False           # flexible CG (automatic with a learned stage)
    # "jacobi" | "chebyshev" (same sweep count, polynomial on [lambda/cheb_ratio, lambda];
    # needs omega_mode="auto", n_smooth <= 2)
    smoother: str = "jacobi"
    cheb_ratio: int = 30
    autotune: bool = True            # time z-chunk candidates of the marching kernels at set-up
    omega_mode: str = "fixed"        # "fixed" (reference) | "auto" (omega_l = rel * 2 / lambda_l)
    omega_rel: float = 0.8
    power_iters: int = 20
    fine_kernel: str = "modal"       # "modal" (z-marching, TMA) | "modal_cpasync" | "gather" (27-neighbour)
    modal_zchunk: int = 0            # z-planes per CTA of the modal kernel (0 = automatic, -1 = one even wave)
    coarse_storage: str = "sym_half"  # Galerkin stencils: "sym_half" | "sym" | "full"
    # bit l: the transfer from Galerkin level l to l+1 uses the smoothed
    # prolongation (I - (4/3) D^-1 A_l / lambda_l) P; bit 1 (level 1 -> 2) only
    smoothed_transfers: int = 0
    smoothed_level_sweeps: int = 0   # sweeps on a level whose transfer down is smoothed (0: n_smooth)
    learned_watch: int = 64          # learned stage: iterations without halving the residual before
                                     # the stage is switched off and plain PCG takes over (0: never)

    @classmethod
    def reference(cls, **kw):
        """The reference algorithm, FP64 (core/multigrid.py)."""
        return cls(**kw)

    @classmethod
    def robust(cls, **kw):
        """FP64 Galerkin hierarchy with a direct coarsest solve ("plain GMG-PCG").

        The reference's stall guard (5x above the best ratio after 10
        iterations) is off: it was tuned for the rediscretized hierarchy, and
        the CG residual norm of a converging solve on high-contrast geometry is
        not monotone."""
        base = dict(coarse="galerkin", coarsest="cholesky", omega_mode="auto", stall_guard=False,
                    smoother=_preset_smoother(kw), smoothed_transfers=_preset_transfers(kw),
                    smoothed_level_sweeps=_preset_level_sweeps(kw))
        base.update(kw)
        return cls(**base)

    @classmethod
    def fast(cls, **kw):
        """Galerkin hierarchy, mixed precision: by default FP64 PCG preconditioned by
        the FP32 V-cycle (``mixed_mode="outer64"``)."""
        base = dict(coarse="galerkin", coarsest="cholesky", precision="mixed", omega_mode="auto",
                    stall_guard=False, smoother=_preset_smoother(kw), smoothed_transfers=_preset_transfers(kw),
                    smoothed_level_sweeps=_preset_level_sweeps(kw))
        base.update(kw)
        return cls(**base)


def _node_dims(nx, ny, nz):
    return (nx + 1, ny + 1, nz + 1)


def _injected_free(levels, fixed_dofs):
    """Per-level free masks by injection (core/multigrid.py:255-278); host
    bookkeeping only, for the ``levels[li]['free']`` attribute."""
    free0 = np.ones(levels[0]["ndof"], dtype=bool)
    fd = np.asarray(fixed_dofs, dtype=np.int64)
    if fd.size:
        free0[fd] = False
    levels[0]["free"] = free0
    prev, prev_dims = free0, _node_dims(*levels[0]["dims"])
    for li in range(1, len(levels)):
        Lcx, Lcy, Lcz = _node_dims(*levels[li]["dims"])
        Lfx, Lfy, _ = prev_dims
        n = np.arange(Lcx * Lcy * Lcz)
        fid = 2 * (n % Lcx) + Lfx * (2 * ((n // Lcx) % Lcy) + Lfy * (2 * (n // (Lcx * Lcy))))
        free = np.ones(3 * n.size, dtype=bool)
        for c in range(3):
            free[3 * n + c] = prev[3 * fid + c]
        levels[li]["free"] = free
        prev, prev_dims = free, (Lcx, Lcy, Lcz)


class MGSolver:
    """Multigrid-preconditioned CG on the full voxel grid, on the B200."""

    _TRY_POOLED_SMOOTH = False   # reference class switch (multigrid.py:83); no pools here

    def __init__(self, nx, ny, nz, fixed_dofs, nu=0.3, xp=None, n_smooth=2, omega=0.6,
                 min_elems=4, max_levels=6, compute_mode="AUTO", cpu_threads=0,
                 verbose=False, options=None, method=_lib.VF_METHOD_MG):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nelem = nx * ny * nz
        self.ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
        self.n_smooth = n_smooth
        self.omega = omega
        self.nu = nu
        self.verbose = verbose
        self.options = options if options is not None else SolverOptions()
        self.xp = np
        self.plan = compute_plan.choose(self.ndof, mode=compute_mode, cpu_threads=cpu_threads,
                                        verbose=verbose)
        self._h = None
        L = _lib.load()
        o = _lib.default_options()
        o.method = method
        o.precision = _lib.PRECISIONS[self.options.precision]
        o.n_smooth = int(n_smooth)
        o.omega = float(omega)
        o.min_elems = int(min_elems)
        o.max_levels = int(max_levels)
        o.coarse_op = _lib.COARSE_OPS[self.options.coarse]
        o.coarsest = _lib.COARSEST[self.options.coarsest]
        o.coarse_sweeps = int(self.options.coarse_sweeps)
        o.stall_guard = int(bool(self.options.stall_guard))
        o.check_every = int(self.options.check_every)
        o.use_graphs = int(bool(self.options.use_graphs))
        o.device = int(self.options.device)
        o.inner_tol = float(self.options.inner_tol)
        o.max_outer = int(self.options.max_outer)
        o.omega_mode = {"fixed": _lib.VF_OMEGA_FIXED, "auto": _lib.VF_OMEGA_AUTO}[self.options.omega_mode]
        o.omega_rel = float(self.options.omega_rel)
        o.power_iters = int(self.options.power_iters)
        o.fine_kernel = {"modal": _lib.VF_FINE_MODAL, "gather": _lib.VF_FINE_GATHER,
                         "modal_cpasync": _lib.VF_FINE_MODAL_CPASYNC}[self.options.fine_kernel]
        o.modal_zchunk = int(self.options.modal_zchunk)
        o.coarse_storage = _lib.STENCIL_STORAGE[self.options.coarse_storage]
        o.mixed_mode = _lib.MIXED_MODES[self.options.mixed_mode]
        o.flexible = int(bool(self.options.flexible))
        o.autotune = int(bool(self.options.autotune))
        o.smoother = _lib.SMOOTHERS[self.options.smoother]
        o.cheb_ratio = int(self.options.cheb_ratio)
        o.smoothed_transfers = int(self.options.smoothed_transfers)
        o.learned_watch = int(self.options.learned_watch)
        o.smoothed_level_sweeps = int(self.options.smoothed_level_sweeps)
        h = ctypes.c_void_p()
        _lib.check(L.vf_create(int(nx), int(ny), int(nz), float(nu), ctypes.byref(o), ctypes.byref(h)),
                   None, "vf_create")
        self._h = h
        n = ctypes.c_int32()
        L.vf_num_levels(h, ctypes.byref(n))
        self.levels = []
        d3 = (ctypes.c_int32 * 3)()
        for li in range(n.value):
            L.vf_level_dims(h, li, d3)
            lx, ly, lz = int(d3[0]), int(d3[1]), int(d3[2])
            self.levels.append({"dims": (lx, ly, lz), "ndof": 3 * (lx + 1) * (ly + 1) * (lz + 1),
                                "g": float(2 ** li), "free": None})
        self.last_iters = 0
        self.last_converged = None
        self.last_resid_ratio = float("nan")
        self.resid_history = []
        self.last_info = None
        self._density_set = False
        self._build_free(fixed_dofs)

    # -- lifetime ------------------------------------------------------------
    def close(self):
        """Release the device state (core/multigrid.py:245-252)."""
        if self._h is not None:
            _lib.load().vf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _handle(self):
        if self._h is None:
            raise RuntimeError("solver is closed")
        return self._h

    # -- boundary conditions / density -----------------------------------------
    def _build_free(self, fixed_dofs):
        fd = np.ascontiguousarray(np.asarray(fixed_dofs, dtype=np.int64).ravel())
        self._fixed = fd
        _lib.check(_lib.load().vf_set_fixed(self._handle(), _lib.ptr(fd), fd.size), self._h,
                   "set_fixed")
        if self.options.coarse == "rediscretize":
            _injected_free(self.levels, fd)
        else:
            _injected_free(self.levels[:1], fd)
        self._density_set = False

    def set_density(self, Evec_full, nu_elem=None):
        """Per-element modulus (core/multigrid.py:281-315): builds every
        level's operator and diagonal on the device.  ``nu_elem`` optionally
        gives a per-voxel Poisson ratio (B200 extension)."""
        E = _lib.f64(np.asarray(Evec_full, dtype=float).ravel())
        if E.size != self.nelem:
            raise ValueError(f"Evec has {E.size} entries, expected {self.nelem}")
        nu_e = None if nu_elem is None else _lib.f64(np.asarray(nu_elem, dtype=float).ravel())
        _lib.check(_lib.load().vf_set_material(self._handle(), _lib.ptr(E), _lib.ptr(nu_e), 0), self._h,
                   "set_density")
        self._density_set = True

    # -- level operators (reference private API, routed to the device) ------
    def _need_density(self):
        if not self._density_set:
            raise RuntimeError("call set_density() first")

    def _level_call(self, fn, li, *arrays, out_level=None, precision="fp64", extra=()):
        self._need_density()
        out_level = li if out_level is None else out_level
        out = np.empty(self.levels[out_level]["ndof"])
        args = [_lib.ptr(_lib.f64(a)) for a in arrays]
        prec = _lib.PRECISIONS[precision]
        _lib.check(fn(self._handle(), li, prec, *args, *extra, _lib.ptr(out)), self._h)
        return out

    def _apply(self, li, u, precision="fp64"):
        """y = where(free, K_li u, 0) (core/multigrid.py:318-341)."""
        return self._level_call(_lib.load().vf_apply, li, u, precision=precision)

    _apply_pooled = None   # set below: level-0 apply (multigrid.py:343-365)

    def _smooth(self, li, u, b, iters, precision="fp64"):
        """``iters`` damped-Jacobi sweeps (core/multigrid.py:367-402)."""
        self._need_density()
        out = np.empty(self.levels[li]["ndof"])
        u = _lib.f64(u)
        b = _lib.f64(b)
        _lib.check(_lib.load().vf_smooth(self._handle(), li, _lib.PRECISIONS[precision], _lib.ptr(u),
                                         _lib.ptr(b), int(iters), _lib.ptr(out)), self._h)
        return out

    def _restrict(self, li, r_fine, precision="fp64"):
        """R = P^T then coarse mask (core/multigrid.py:404-416)."""
        return self._level_call(_lib.load().vf_restrict, li, r_fine, out_level=li + 1,
                                precision=precision)

    def _prolongate(self, li, e_coarse, precision="fp64"):
        """where(free_f, P e_c) (core/multigrid.py:418-424)."""
        return self._level_call(_lib.load().vf_prolongate, li, e_coarse, precision=precision)

    def _vcycle(self, li, b, precision="fp64"):
        """One V-cycle from level 0 (core/multigrid.py:426-436)."""
        if li != 0:
            raise ValueError("the device V-cycle starts at level 0")
        self._need_density()
        out = np.empty(self.ndof)
        b = _lib.f64(b)
        _lib.check(_lib.load().vf_vcycle(self._handle(), _lib.PRECISIONS[precision], _lib.ptr(b),
                                         _lib.ptr(out)), self._h)
        return out

    def level_omega(self, li):
        """(omega, lambda_max estimate) of level li after set_density."""
        w = ctypes.c_double()
        lam = ctypes.c_double()
        _lib.check(_lib.load().vf_level_omega(self._handle(), li, ctypes.byref(w), ctypes.byref(lam)), self._h)
        return w.value, lam.value

    def inv_diagonal(self, li):
        """levels[li]['Minv'] (core/multigrid.py:300-304), 3 values per node."""
        self._need_density()
        out = np.empty(self.levels[li]["ndof"])
        _lib.check(_lib.load().vf_inv_diagonal(self._handle(), li, _lib.ptr(out)), self._h)
        return out

    # -- public solve ------------------------------------------------------------
    def solve(self, Evec_full, f, tol=1e-4, max_cg=None, x0=None, progress_cb=None, nu_elem=None, out=None):
        """PCG with the V-cycle preconditioner; returns a fresh numpy u
        (core/multigrid.py:439-583).  ``progress_cb(it, resid_ratio, tol)`` is
        called once per iteration, in order (bursts at graph-chunk ends).
        ``out`` (B200 extension): a C-contiguous float64 array of ndof values
        that receives u and is returned (e.g. page-locked host memory, which
        the device writes at full PCIe / C2C speed)."""
        self.resid_history = []
        t0 = time.perf_counter()
        self.set_density(Evec_full, nu_elem=nu_elem)
        f = _lib.f64(np.asarray(f, dtype=float).ravel())
        if f.size != self.ndof:
            raise ValueError(f"f has {f.size} entries, expected {self.ndof}")
        x0a = None if x0 is None else _lib.f64(np.asarray(x0, dtype=float).ravel())
        if out is not None:
            if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.size != self.ndof
                    or not out.flags.c_contiguous):
                raise ValueError(f"out must be a C-contiguous float64 array of {self.ndof} values")
            u = out if out.ndim == 1 else out.reshape(-1)   # a view of out either way
        else:
            u = np.empty(self.ndof)
        info = _lib.VfSolveInfo()
        cb_error = []

        def _tramp(it, resid, tl, _user):
            if progress_cb is None or cb_error:
                return
            try:
                progress_cb(int(it), float(resid), float(tl))
            except BaseException as exc:  # noqa: BLE001  re-raised after the call
                cb_error.append(exc)

        cfun = _lib.PROGRESS_FN(_tramp)
        L = _lib.load()
        rc = L.vf_solve_cb(self._handle(), _lib.ptr(f), _lib.ptr(x0a), float(tol),
                           int(max_cg or 0), 0, _lib.ptr(u), ctypes.byref(info), cfun, None)
        self.last_info = info
        if rc not in (_lib.VF_OK, _lib.VF_ERR_STALLED):
            _lib.check(rc, self._h, "solve")
        if info.iters < 0:
            u[:] = 0.0                   # zero load (multigrid.py:471-473)
            return u
        n = ctypes.c_int32()
        L.vf_resid_history(self._h, None, 0, ctypes.byref(n))
        hist = np.empty(n.value)
        L.vf_resid_history(self._h, _lib.ptr(hist), n.value, ctypes.byref(n))
        self.resid_history = [float(v) for v in hist]
        self.last_iters = int(info.iters)
        self.last_converged = bool(info.converged)
        self.last_resid_ratio = float(info.resid_ratio)
        if cb_error:
            raise cb_error[0]
        if rc == _lib.VF_ERR_STALLED:
            _lib.check(rc, self._h)
        if not self.last_converged:
            print(f"[VoxelSim FEA] WARNING: MG-PCG did not converge in {max_cg or 1000} "
                  f"iterations (tol={tol:g}, final residual ratio={self.last_resid_ratio:.3e}, "
                  f"plan={self.plan.label}). Returned displacement may be inaccurate.")
        if self.verbose:
            print(f"[VoxelSim FEA] MG solve: {self.last_iters} CG iters "
                  f"(converged={self.last_converged}), total={(time.perf_counter() - t0) * 1e3:.1f}ms | "
                  f"device={info.device_ms:.1f}ms setup={info.setup_ms:.1f}ms "
                  f"true residual={info.true_resid:.3e}")
        return u


def _solve_block(self, Evec_full, F, tol=1e-4, max_cg=None, nu_elem=None):
    """k load cases on one geometry as one call (B200 extension; the reference
    calls ``solve`` once per case): F is (k, ndof); returns U (k, ndof).  The
    cases share the operator set-up and run concurrently on the device.
    Per-case results land in ``last_block_info`` (k vf_solve_info records)."""
    self.set_density(Evec_full, nu_elem=nu_elem)
    F = np.ascontiguousarray(np.asarray(F, dtype=float).reshape(-1, self.ndof))
    k = F.shape[0]
    U = np.empty_like(F)
    infos = (_lib.VfSolveInfo * k)()
    rc = _lib.load().vf_solve_block(self._handle(), _lib.ptr(F), k, float(tol), int(max_cg or 0), 0,
                                    _lib.ptr(U), infos)
    self.last_block_info = list(infos)
    if rc not in (_lib.VF_OK, _lib.VF_ERR_STALLED):
        _lib.check(rc, self._h, "solve_block")
    self.last_iters = max(int(i.iters) for i in infos)
    self.last_converged = all(bool(i.converged) for i in infos)
    if rc == _lib.VF_ERR_STALLED:
        _lib.check(rc, self._h)
    return U


MGSolver.solve_block = _solve_block


def solve_batch(solvers, E_list, F_list, tol=1e-4, max_cg=None, nu_list=None):
    """Independent parts in one call (B200 extension): solver i gets E_list[i]
    (and nu_list[i]) and F_list[i]; all parts are set up and solved
    concurrently.  Returns the list of displacements; per-part results land in
    each solver's ``last_info``."""
    n = len(solvers)
    P = ctypes.c_void_p
    Es = [_lib.f64(np.asarray(e, dtype=float).ravel()) for e in E_list]
    Fs = [_lib.f64(np.asarray(f, dtype=float).ravel()) for f in F_list]
    Ns = None if nu_list is None else [None if v is None else _lib.f64(np.asarray(v, dtype=float).ravel())
                                       for v in nu_list]
    Us = [np.empty(s.ndof) for s in solvers]
    for s, e, f in zip(solvers, Es, Fs):
        if e.size != s.nelem or f.size != s.ndof:
            raise ValueError("batch: E / F sizes do not match the solver grids")
    h = (P * n)(*[s._handle() for s in solvers])
    e_arr = (P * n)(*[e.ctypes.data for e in Es])
    n_arr = None if Ns is None else (P * n)(*[None if v is None else v.ctypes.data for v in Ns])
    f_arr = (P * n)(*[f.ctypes.data for f in Fs])
    u_arr = (P * n)(*[u.ctypes.data for u in Us])
    infos = (_lib.VfSolveInfo * n)()
    rc = _lib.load().vf_solve_batch(h, n, e_arr, n_arr, f_arr, float(tol), int(max_cg or 0), 0, u_arr, infos)
    for s, i in zip(solvers, infos):
        s.last_info = i
        s.last_iters = int(i.iters)
        s.last_converged = bool(i.converged)
        s._density_set = True
    if rc != _lib.VF_OK:
        raise RuntimeError(f"solve_batch failed: {_lib.load().vf_global_last_error().decode()}")
    return Us
MGSolver._apply_pooled = lambda self, u: self._apply(0, u)
