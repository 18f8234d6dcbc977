"""The out-of-process solve job on the B200 -- a drop-in for VoxelSim-FEA
core/solve_worker.py: same ``SolverClient`` (start / poll / cancel /
cleanup), same ``job.pkl`` input, same ``status.json`` phases
(voxel -> solve -> done | error) and the same ``final.pkl`` keys, so the
add-on's parent side runs unchanged.

What runs where: the inside tests of the part / exclusion / bearing / load
meshes on the device (voxelsim_fea_b200.inside: the reference's parity ray
cast, points generated on the device); grid assembly on the host (O(voxels)
bookkeeping, solve_worker.py:242-287); the unsupported-island removal, the
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


class SolverClient:
    """Launch the worker and poll it without blocking (solve_worker.py:46-167).

    Events from :meth:`poll`: ('voxel', frac), ('solve', info|None),
    ('done', final dict), ('error', message), ('running', frac)."""

    def __init__(self):
        self._proc = None
        self._dir = None
        self._logf = None
        self._finished = False

    def start(self, job):
        self._dir = tempfile.mkdtemp(prefix="voxfea_b200_solve_")
        job_path = os.path.join(self._dir, "job.pkl")
        with open(job_path, "wb") as fh:
            pickle.dump(job, fh)
        cmd = [sys.executable, "-m", "voxelsim_fea_b200.solve_worker", job_path, self._dir]
        env = dict(os.environ)
        pkg_parent = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        env["PYTHONPATH"] = os.pathsep.join(p for p in (pkg_parent, env.get("PYTHONPATH", "")) if p)
        self._logf = open(os.path.join(self._dir, "worker.log"), "wb")
        self._proc = subprocess.Popen(cmd, stdout=self._logf, stderr=self._logf, env=env)

    def _status(self):
        try:
            with open(os.path.join(self._dir, "status.json")) as fh:
                return json.load(fh)
        except Exception:
            return None

    def _log_tail(self):
        try:
            with open(os.path.join(self._dir, "worker.log"), "rb") as fh:
                return fh.read().decode("utf-8", "replace").strip()
        except Exception:
            return ""

    def poll(self):
        if self._finished:
            return ("running", 1.0)
        st = self._status()
        if st is None:
            if self._proc is not None and self._proc.poll() is not None:
                return ("error", self._log_tail() or "worker exited early")
            return ("running", 0.0)
        phase = st.get("phase")
        if phase == "error":
            return ("error", st.get("error") or self._log_tail() or "worker error")
        if phase == "voxel":
            return ("voxel", float(st.get("frac", 0.0)))
        if phase == "solve":
            info = None
            if "cg_iter" in st:
                info = {"iter": int(st.get("cg_iter", 0)), "resid": float(st.get("cg_resid", float("nan"))),
                        "tol": float(st.get("cg_tol", 1e-6))}
            return ("solve", info)
        if phase == "done":
            try:
                with open(os.path.join(self._dir, "final.pkl"), "rb") as fh:
                    final = pickle.load(fh)
            except Exception as exc:
                return ("error", f"could not read solver result: {exc}")
            self._finished = True
            return ("done", final)
        return ("running", 0.0)

    def wait(self, timeout=None, interval=0.05):
        """Block until done/error (convenience for scripts and tests)."""
        t0 = time.time()
        while True:
            ev = self.poll()
            if ev[0] in ("done", "error"):
                return ev
            if timeout is not None and time.time() - t0 > timeout:
                return ("error", "timeout")
            time.sleep(interval)

    def cancel(self):
        if self._proc is not None and self._proc.poll() is None:
            try:
                self._proc.terminate()
            except Exception:
                pass
        self.cleanup()

    def cleanup(self):
        if self._logf is not None:
            try:
                self._logf.close()
            except Exception:
                pass
            self._logf = None
        if self._dir and os.path.isdir(self._dir):
            shutil.rmtree(self._dir, ignore_errors=True)
        self._dir = None


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
    """Grid assembly (solve_worker.py:242-270): active voxels, fixed DOFs,
    nodal force vector from the role masks."""
    nx, ny, nz = dims
    inside = None
    excl = np.zeros(nx * ny * nz, dtype=bool)
    fixed = []
    force = np.zeros(3 * (nx + 1) * (ny + 1) * (nz + 1))
    for (role, meta), mask in zip(descr, masks):
        if role == "build":
            inside = mask
        elif role == "exclude":
            excl = excl | mask
        elif role == "bearing":
            nodes = np.nonzero(mask)[0]
            for c, on in enumerate(meta):
                if on:
                    fixed.append(3 * nodes + c)
        elif role == "load":
            nodes = np.nonzero(mask)[0]
            if len(nodes):
                fv = np.asarray(meta, dtype=float) / len(nodes)
                for c in range(3):
                    force[3 * nodes + c] += fv[c]
    if inside is None:
        inside = np.zeros(nx * ny * nz, dtype=bool)
    active = inside & ~excl
    fixed_dofs = np.unique(np.concatenate(fixed)).astype(np.int64) if fixed else np.zeros(0, dtype=np.int64)
    return active, fixed_dofs, force


def _worker_main(job_path, work_dir):
    from . import fea, inside
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
    active, fixed_dofs, force = assemble(descr, masks, dims)
    n_islands_removed = 0
    if fixed_dofs.size and active.any():
        kept3d, n_islands_removed = fea.drop_unsupported_islands(active.reshape(nx, ny, nz), fixed_dofs)
        if n_islands_removed:
            active = kept3d.ravel()
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
