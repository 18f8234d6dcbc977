"""The out-of-process solve job on the B200 -- a drop-in for VoxelSim-FEA
core/solve_worker.py: same ``SolverClient`` (start / poll / cancel /
cleanup), same ``job.pkl`` input, same ``status.json`` phases
(voxel -> solve -> done | error) and the same ``final.pkl`` keys, so the
add-on's parent side runs unchanged.

What runs where: the inside tests of the part / exclusion / bearing / load
meshes on the device (voxelsim_fea_b200.inside: the reference's parity ray
cast, points generated on the device); grid assembly on the device
(vf_assemble_grid: active voxels, fixed-DOF bits, nodal forces,
solve_worker.py:242-287); the unsupported-island removal, the
solve and the von Mises stress on the device (VoxelFEA); the per-element
displacement / safety-factor fields and the summary numbers as in
solve_worker.py:356-431.

One job key beyond the reference's: ``"solver": "reference"`` runs the
reference's own multigrid algorithm (rediscretized levels, omega 0.6) instead
of the default robust hierarchy; the solution is the same to the solver
tolerance, the iteration count and history are then the reference's.
"""

import json
import os
import pickle
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

_STRESS_PERCENTILE = 99.0   # solve_worker.py:37


class _JobFiles:
    """The files one job exchanges with its worker, in a private temp folder:
    job.pkl (in), status.json (progress, rewritten atomically by the worker),
    final.pkl (result) and worker.log (the worker's stdout and stderr)."""

    def __init__(self):
        self.root = tempfile.mkdtemp(prefix="voxfea_b200_solve_")
        self.job = os.path.join(self.root, "job.pkl")
        self.status = os.path.join(self.root, "status.json")
        self.final = os.path.join(self.root, "final.pkl")
        self.log = os.path.join(self.root, "worker.log")

    def spawn_worker(self, job):
        """Write the job and start the worker process on it; returns
        (process, open log handle)."""
        with open(self.job, "wb") as fh:
            pickle.dump(job, fh)
        # the worker imports this package by name: put its parent folder on the
        # child's path (the parent process's own sys.path is left alone)
        env = os.environ.copy()
        here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        env["PYTHONPATH"] = os.pathsep.join(filter(None, [here, env.get("PYTHONPATH")]))
        log = open(self.log, "wb")
        proc = subprocess.Popen([sys.executable, "-m", "voxelsim_fea_b200.solve_worker", self.job, self.root],
                                stdout=log, stderr=subprocess.STDOUT, env=env)
        return proc, log

    def read_status(self):
        """The worker's last status record, or None while there is none (or
        it cannot be parsed yet)."""
        try:
            with open(self.status) as fh:
                return json.load(fh)
        except (OSError, ValueError):
            return None

    def read_final(self):
        with open(self.final, "rb") as fh:
            return pickle.load(fh)

    def log_text(self):
        try:
            with open(self.log, "rb") as fh:
                return fh.read().decode("utf-8", "replace").strip()
        except OSError:
            return ""

    def remove(self):
        shutil.rmtree(self.root, ignore_errors=True)


class SolverClient:
    """Runs one solve job in a worker process and reports its progress without
    blocking -- the parent side of core/solve_worker.py (its SolverClient,
    solve_worker.py:44-153), whose event protocol this keeps.

    :meth:`poll` returns one of
      ('voxel', frac)    the worker is building the grid (0..1);
      ('solve', info)    the CG solve runs; info is None until the worker's
                         first progress record, then {'iter', 'resid', 'tol'};
      ('done', final)    the result dict of final.pkl (returned once; later
                         polls give ('running', 1.0));
      ('error', message)
      ('running', frac)  nothing new to report."""

    def __init__(self):
        self._files = None
        self._proc = None
        self._log = None
        self._delivered = False

    def start(self, job):
        self._files = _JobFiles()
        self._proc, self._log = self._files.spawn_worker(job)

    # -- progress ------------------------------------------------------------
    def poll(self):
        if self._delivered:
            return ("running", 1.0)
        status = self._files.read_status() if self._files is not None else None
        if status is None:
            return self._before_first_status()
        react = self._BY_PHASE.get(status.get("phase"))
        return react(self, status) if react is not None else ("running", 0.0)

    def _before_first_status(self):
        exited = self._proc is not None and self._proc.poll() is not None
        if exited:
            log = self._files.log_text() if self._files is not None else ""
            return ("error", log or "worker exited early")
        return ("running", 0.0)

    def _phase_voxel(self, status):
        return ("voxel", float(status.get("frac", 0.0)))

    def _phase_solve(self, status):
        if "cg_iter" not in status:
            return ("solve", None)
        return ("solve", {"iter": int(status["cg_iter"]),
                          "resid": float(status.get("cg_resid", float("nan"))),
                          "tol": float(status.get("cg_tol", 1e-6))})

    def _phase_done(self, status):
        try:
            final = self._files.read_final()
        except Exception as exc:   # a truncated or missing result file
            return ("error", f"could not read solver result: {exc}")
        self._delivered = True
        return ("done", final)

    def _phase_error(self, status):
        return ("error", status.get("error") or self._files.log_text() or "worker error")

    _BY_PHASE = {"voxel": _phase_voxel, "solve": _phase_solve, "done": _phase_done, "error": _phase_error}

    def wait(self, timeout=None, interval=0.05):
        """Poll until the job is done or failed (for scripts and tests)."""
        deadline = None if timeout is None else time.monotonic() + timeout
        while True:
            event = self.poll()
            if event[0] in ("done", "error"):
                return event
            if deadline is not None and time.monotonic() > deadline:
                return ("error", "timeout")
            time.sleep(interval)

    # -- teardown --------------------------------------------------------------
    def cancel(self):
        """Stop a running worker and remove the job's files."""
        if self._proc is not None and self._proc.poll() is None:
            self._proc.terminate()
        self.cleanup()

    def cleanup(self):
        """Close the log handle and remove the job's files (idempotent)."""
        log, self._log = self._log, None
        if log is not None and not log.closed:
            log.close()
        files, self._files = self._files, None
        if files is not None:
            files.remove()


def solver_available():
    try:
        from . import _lib
        _lib.load()
        return bool(sys.executable)
    except Exception:
        return False


def _atomic_write(path, data, mode):
    tmp = path + ".tmp"
    with open(tmp, mode) as fh:
        if mode == "w":
            json.dump(data, fh)
        else:
            pickle.dump(data, fh)
    for i in range(10):   # readers may hold the destination open briefly
        try:
            os.replace(tmp, path)
            return
        except PermissionError:
            time.sleep(0.05 * (i + 1))
    os.replace(tmp, path)


def element_displacement(u, dims):
    """Mean corner displacement magnitude per voxel, on the device
    (vf_element_displacement; solve_worker.py:374-388)."""
    import ctypes
    from . import _lib
    nx, ny, nz = (int(v) for v in dims)
    uu = _lib.f64(np.asarray(u, dtype=float).ravel())
    out = np.empty(nx * ny * nz, dtype=np.float32)
    _lib.check(_lib.load().vf_element_displacement(nx, ny, nz, _lib.ptr(uu), out.ctypes.data_as(ctypes.c_void_p)),
               None, "element_displacement")
    return out


def assemble(descr, masks, dims):
    """Grid assembly (solve_worker.py:242-270) on the device (vf_assemble_grid):
    role masks -> (active bool[nelem], fixed_dofs int64 sorted, force
    float64[ndof], fixed_bits uint8[nnode] with bit c set <=> DOF c fixed)."""
    import ctypes
    from . import _lib
    nx, ny, nz = (int(v) for v in dims)
    ne, nn = nx * ny * nz, (nx + 1) * (ny + 1) * (nz + 1)
    n = len(descr)
    roles = np.array([_lib.ROLES[r] for r, _ in descr], dtype=np.int32)
    meta = np.zeros(3 * max(n, 1))
    arrays = []
    for i, ((role, m), mask) in enumerate(zip(descr, masks)):
        size = ne if role in ("build", "exclude") else nn
        a = np.ascontiguousarray(np.asarray(mask, dtype=bool).ravel().view(np.uint8))
        if a.size != size:
            raise ValueError(f"{role} mask has {a.size} entries, expected {size}")
        arrays.append(a)
        if role in ("bearing", "load"):
            meta[3 * i:3 * i + 3] = np.asarray(m, dtype=float)[:3]
    ptrs = (ctypes.c_void_p * max(n, 1))(*[a.ctypes.data for a in arrays])
    active = np.empty(ne, dtype=np.uint8)
    bits = np.empty(nn, dtype=np.uint8)
    force = np.empty(3 * nn)
    n_act, n_fix = ctypes.c_int64(), ctypes.c_int64()
    _lib.check(_lib.load().vf_assemble_grid(nx, ny, nz, n, _lib.ptr(roles), ptrs, _lib.ptr(meta), 0,
                                            _lib.ptr(active), _lib.ptr(bits), _lib.ptr(force),
                                            ctypes.byref(n_act), ctypes.byref(n_fix)), None, "assemble")
    fixed_dofs = np.flatnonzero(((bits[:, None] >> np.arange(3, dtype=np.uint8)) & 1).ravel()).astype(np.int64)
    return active.astype(bool), fixed_dofs, force, bits


def drop_unsupported_islands_bits(active, fixed_bits, dims):
    """Island removal (core/fea.py:207-227) with the supports as per-node
    fixed-DOF bits, on the device; returns (kept bool[nelem], n_removed)."""
    import ctypes
    from . import _lib
    nx, ny, nz = (int(v) for v in dims)
    act = np.ascontiguousarray(np.asarray(active, dtype=bool).ravel().view(np.uint8))
    kept = np.empty_like(act)
    nrem = ctypes.c_int64()
    _lib.check(_lib.load().vf_drop_unsupported_islands_mask(nx, ny, nz, _lib.ptr(act),
                                                            _lib.ptr(np.ascontiguousarray(fixed_bits)), 0,
                                                            _lib.ptr(kept), ctypes.byref(nrem)),
               None, "drop_unsupported_islands")
    return kept.astype(bool), int(nrem.value)


def _worker_main(job_path, work_dir):
    from . import inside
    from .fea import VoxelFEA
    from .multigrid import SolverOptions

    status_path = os.path.join(work_dir, "status.json")

    def set_status(**kw):
        _atomic_write(status_path, kw, "w")

    set_status(phase="voxel", frac=0.0)
    with open(job_path, "rb") as fh:
        job = pickle.load(fh)
    g = job["grid"]
    dims = tuple(int(v) for v in g["dims"])
    origin = np.asarray(g["origin"], dtype=float)
    vsize = float(g["vsize"])
    nx, ny, nz = dims
    direction = job.get("direction")

    # --- inside tests on the device ------------------------------------------
    queries, descr = job["queries"], job["descr"]
    npts = {"centers": nx * ny * nz, "nodes": (nx + 1) * (ny + 1) * (nz + 1)}
    total = sum(npts[q["target"]] for q in queries) or 1
    done, masks = 0, []
    for q in queries:
        masks.append(inside.inside_grid(q["verts"], q["faces"], dims, origin, vsize, q["target"], direction))
        done += npts[q["target"]]
        set_status(phase="voxel", frac=done / total)

    # --- grid assembly, islands ------------------------------------------------
    active, fixed_dofs, force, fixed_bits = assemble(descr, masks, dims)
    n_islands_removed = 0
    if fixed_dofs.size and active.any():
        kept, n_islands_removed = drop_unsupported_islands_bits(active, fixed_bits, dims)
        if n_islands_removed:
            active = kept
    if int(active.sum()) == 0:
        set_status(phase="error", error="No material inside the part at this resolution "
                                        "(check the Part object / resolution)")
        return
    if fixed_dofs.size == 0:
        set_status(phase="error", error="No supports (bearings) reach any grid node at this resolution -- "
                                        "move/enlarge the support mesh or raise the resolution")
        return
    if not np.any(force):
        set_status(phase="error", error="No load reaches any grid node -- check the Load mesh(es) and "
                                        "force vector(s)")
        return

    # --- the solve -------------------------------------------------------------
    set_status(phase="solve", frac=0.0)
    mat = job["material"]
    E = float(mat["youngs_modulus"])
    nu = float(mat["poisson"])
    yield_strength = float(mat.get("yield_strength") or 0.0)
    active3d = active.reshape(nx, ny, nz)
    nelem = nx * ny * nz
    mg_options = SolverOptions() if job.get("solver") == "reference" else None
    vfea = VoxelFEA(nx, ny, nz, nu=nu, active_elems=active3d, compute_mode=job.get("compute_mode", "AUTO"),
                    cpu_threads=int(job.get("cpu_threads", 0)), verbose=bool(job.get("verbose", False)),
                    mg_options=mg_options)
    last = [0.0]

    def _cg_progress(it, resid_ratio, tol):
        now = time.time()
        if now - last[0] < 0.15:
            return
        last[0] = now
        set_status(phase="solve", frac=0.0, cg_iter=it, cg_resid=resid_ratio, cg_tol=tol)

    try:
        vfea.set_fixed(fixed_dofs)
        # unit-cube Ke: stiffness modulus E*vsize, stress with E then / vsize (solve_worker.py:338-355)
        u_full = vfea.solve(np.full(nelem, E * vsize), force, tol=1e-6, progress_cb=_cg_progress)
        vm = vfea.element_von_mises_stress(u_full, np.full(nelem, E)) / vsize
    finally:
        resid_history = list(vfea.resid_history)
        vfea.close()

    # --- result fields (solve_worker.py:360-431) ---------------------------------
    active_vals = vm[active]
    max_stress_pa = float(active_vals.max()) if active_vals.size else 0.0
    scale_vmax = float(np.percentile(active_vals, _STRESS_PERCENTILE)) if active_vals.size else 0.0
    scale_vmax = max(scale_vmax, 1e-6)
    disp_mag = np.sqrt((u_full.reshape(-1, 3) ** 2).sum(axis=1))
    max_disp_m = float(disp_mag.max()) if disp_mag.size else 0.0
    disp3d = element_displacement(u_full, dims).reshape(nx, ny, nz).astype(float)
    safety_cap = 10.0
    safety3d = np.zeros(nelem)
    min_safety_factor = None
    if yield_strength > 0 and active_vals.size:
        eps = max(1e-9, 1e-9 * yield_strength)
        ratio = yield_strength / np.maximum(active_vals, eps)
        min_safety_factor = float(ratio.min())
        safety3d[active] = np.clip(ratio, 0.0, safety_cap)
    disp_vmax = max(float(disp3d[active3d].max()) if active3d.any() else 0.0, 1e-9)
    bbox_diag_m = float(np.sqrt(((np.asarray(dims) * vsize) ** 2).sum()))
    reliable = bool(vfea.last_converged) and max_disp_m <= 0.5 * bbox_diag_m
    final = {
        "dims": dims, "origin": origin, "vsize": vsize,
        "active3d": active3d,
        "stress3d": vm.reshape(nx, ny, nz).astype(np.float32),
        "stress_vmax": scale_vmax,
        "max_stress_pa": max_stress_pa,
        "safety3d": safety3d.reshape(nx, ny, nz).astype(np.float32),
        "safety_cap": safety_cap,
        "min_safety_factor": min_safety_factor,
        "yield_strength_pa": yield_strength,
        "displacement3d": disp3d.astype(np.float32),
        "displacement_vmax_m": disp_vmax,
        "max_displacement_m": max_disp_m,
        "cg_iters": int(vfea.last_iters),
        "cg_converged": bool(vfea.last_converged),
        "cg_resid_history": resid_history,
        "cg_tol": 1e-6,
        "reliable": reliable,
        "n_islands_removed": int(n_islands_removed),
        "compute_label": vfea.plan.label,
    }
    _atomic_write(os.path.join(work_dir, "final.pkl"), final, "wb")
    set_status(phase="done", frac=1.0)


def _main(argv):
    job_path, work_dir = argv[1], argv[2]
    try:
        _worker_main(job_path, work_dir)
    except Exception as exc:
        import traceback
        try:
            _atomic_write(os.path.join(work_dir, "status.json"),
                          {"phase": "error", "error": f"{exc}\n{traceback.format_exc()}"}, "w")
        except Exception:
            pass
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(_main(sys.argv))
