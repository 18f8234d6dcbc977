#!/usr/bin/env python
"""Benchmark: time-to-1e-8 relative residual of the matrix-free hex8 GMG-PCG
solve, reported as MDOF/s (full-grid DOF / time-to-solution), on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (default): the seeded 256x128x128 noise bracket (Gaussian noise
blurred sigma=4, 50th-percentile threshold, largest 26-connected component;
aluminium E=69 GPa nu=0.33, z=0 face clamped, 5 kN in -z on a 16x16 top
patch), 5-level GMG, e_min=1e-9 voids on the full grid -- 12,830,211 DOF.
A step is one complete solve from the modulus field and load (coarse-operator
set-up included) to a true FP64 relative residual below 1e-8.

`value`  device-resident: inputs already in HBM, CUDA events on the solver's
         stream around K steps, max over ranks.
`e2e`    the public API (MGSolver.solve with host numpy arrays in page-locked
         memory: modulus and load copied in, displacement copied out every
         step).
`impl reference` times the CPU oracle (a numpy restatement of the reference's
         Jacobi-PCG, the reference path that converges on noise geometry) on a
         bounded sample of the same generator, on the host cores.
N > 1 runs independent replicas (one per GPU, no inter-GPU traffic): the
solve does not shard in this build.
"""

import argparse
import ctypes
import hashlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "MDOF/s to 1e-8 relative residual (time-to-solution), matrix-free hex8 GMG-PCG"
UNIT = "MDOF/s"
TOL = 1e-8
REF_TOL = 1e-12      # the FP64 solve the errors are stated against
E_MIN = 1e-9

WORKLOADS = {
    "bracket_256x128x128": dict(shape=(256, 128, 128), seed=0, sigma=4.0, load=5000.0, patch=16,
                                levels=5),
    "bracket_128x64x64": dict(shape=(128, 64, 64), seed=0, sigma=4.0, load=5000.0, patch=16, levels=4),
    "cantilever_64x16x16": dict(cantilever=True, levels=3),
    # large single solve: two-material (steel / ABS by a second blurred-noise
    # threshold, per-voxel E and nu), 6-level GMG, ~101.6 M DOF
    "twomat_512x256x256": dict(twomat=True, shape=(512, 256, 256), seed=0, sigma=4.0, load=5000.0, patch=16,
                               levels=6),
    "twomat_128x64x64": dict(twomat=True, shape=(128, 64, 64), seed=0, sigma=4.0, load=5000.0, patch=16,
                             levels=4),
    # block right-hand sides: the seeded generator at 192^3 with k load cases
    # (generators.load_cases: unit direction uniform on the sphere, 1-10 kN on a
    # random 8x8 top patch); run with --block 16
    "bracket_192": dict(shape=(192, 192, 192), seed=0, sigma=4.0, load=5000.0, patch=16, levels=5),
}
CPU_SAMPLE = dict(shape=(64, 32, 32), seed=0, sigma=4.0, load=5000.0, patch=16)
PORT_NOTE = ("the reference is pure Python/numpy and is not present on the GPU host; its algorithm runs as the "
             "oracle/ restatement, which is pinned to golden vectors generated by importing the reference "
             "(tests/golden/make_golden.py, tests/test_oracle_golden.py)")
DTYPE_MIXED = ("f32 V-cycle with FP16-valued scaled Galerkin stencils on the coarse levels, f64 Krylov "
               "(FP64 fine operator for A p, dots, coarsest Cholesky solve)")


def make_problem(w):
    from voxelsim_fea_b200 import generators
    if w.get("cantilever"):
        return generators.cantilever()
    if w.get("twomat"):
        return generators.two_material_part(shape=w["shape"], seed=w["seed"], sigma=w["sigma"], load_n=w["load"],
                                            patch=w["patch"])
    return generators.bracket(shape=w["shape"], seed=w["seed"], sigma=w["sigma"], load_n=w["load"],
                              patch=w["patch"])


def mg_modulus(p):
    """VoxelFEA's MG convention: inactive voxels carry e_min * E (fea.py:467-469)."""
    return np.where(p["active"], p["E_stiff"], p["E_stiff"] * E_MIN)


def active_nodes(p):
    """Nodes of the active voxels (reference node order, x fastest)."""
    nx, ny, nz = p["dims"]
    a = np.asarray(p["active"], dtype=bool).reshape(nx, ny, nz)
    n = np.zeros((nx + 1, ny + 1, nz + 1), dtype=bool)
    for ox in (0, 1):
        for oy in (0, 1):
            for oz in (0, 1):
                n[ox:ox + nx, oy:oy + ny, oz:oz + nz] |= a
    return n.transpose(2, 1, 0).ravel()


def field_errors(u, vm, u_ref, vm_ref, node_act, elem_act, apply_k=None):
    """Max-abs error over the active nodes (all three components) / max |u_ref|
    there, the same for the element von Mises stress over active voxels, and
    (with apply_k = the FP64 operator) the energy-norm error
    sqrt(e.K e / u_ref.K u_ref).  The max-norm displacement error also sees
    pieces held only through a node or an edge (hinges of the voxel part),
    whose rigid motion the residual barely constrains; stress and energy do
    not."""
    du = np.abs(u - u_ref).reshape(-1, 3)[node_act]
    su = np.abs(u_ref).reshape(-1, 3)[node_act].max()
    dv = np.abs(vm - vm_ref)[elem_act]
    sv = np.abs(vm_ref)[elem_act].max()
    out = {"u_rel_err": float(du.max() / su), "vm_rel_err": float(dv.max() / sv)}
    if apply_k is not None:
        e = u - u_ref
        out["u_energy_rel_err"] = float(np.sqrt(max(e @ apply_k(e), 0.0) / (u_ref @ apply_k(u_ref))))
    return out


def level_sweeps_kw(args):
    """Solver option override for --smoothed-level-sweeps (none: the presets')."""
    v = getattr(args, "smoothed_level_sweeps", None)
    return {} if v is None else {"smoothed_level_sweeps": int(v)}


# DRAM traffic of the roofline kernel comes from an ncu capture summary under
# profiles/, which records the bytes per launch and a hash of the kernel's
# sources; the figure is reported only while the sources still hash the same.
ROOFLINE_SOURCES = ("vf_modal_tma.cu", "vf_modal.cuh", "vf_wait.cuh", "vf_reduce.cuh")
ROOFLINE_SUMMARY = "k_modal_tma_smooth_fp32_bracket256.md"


def kernel_source_sha(files=ROOFLINE_SOURCES):
    h = hashlib.sha256()
    for f in files:
        with open(os.path.join(REPO, "voxelsim_fea_b200", "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def profiled_traffic(summary=ROOFLINE_SUMMARY):
    """(bytes per launch, note): dram read + write bytes of one launch from the
    summary's `dram_bytes_per_launch:` line, if its `source_sha16:` line matches
    the current sources; (None, why) otherwise."""
    path = os.path.join(REPO, "profiles", summary)
    try:
        text = open(path).read()
    except OSError:
        return None, "no ncu summary"
    rec = {}
    for ln in text.splitlines():
        ln = ln.strip().strip("`")
        for key in ("source_sha16:", "dram_bytes_per_launch:"):
            if ln.startswith(key):
                rec[key[:-1]] = ln[len(key):].strip()
    want = kernel_source_sha()
    if rec.get("source_sha16") != want:
        return None, f"ncu summary {summary} predates the current kernel sources (sha {want})"
    try:
        return float(rec["dram_bytes_per_launch"]), f"ncu capture ({summary}, source sha {want})"
    except (KeyError, ValueError):
        return None, f"ncu summary {summary} has no dram_bytes_per_launch line"


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- replicas
def max_over_ranks(value, dist=None, device=None):
    """Max of a per-rank float over the process group (identity without one).
    Every rank calls it at the same point (timing is max over ranks)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------- reference arm
def cpu_sample_solve():
    """One reference-algorithm solve on the bounded CPU sample; returns (seconds, dof, iters)."""
    from oracle import fea as ofea
    from voxelsim_fea_b200 import generators
    p = generators.bracket(shape=CPU_SAMPLE["shape"], seed=CPU_SAMPLE["seed"], sigma=CPU_SAMPLE["sigma"],
                           load_n=CPU_SAMPLE["load"], patch=CPU_SAMPLE["patch"])
    nx, ny, nz = p["dims"]
    v = ofea.VoxelFEAOracle(nx, ny, nz, nu=p["nu"], active_elems=p["active"], use_multigrid=False)
    v.set_fixed(p["fixed_dofs"])
    t0 = time.perf_counter()
    v.solve(p["E_stiff"], p["f"], tol=TOL)
    dt = time.perf_counter() - t0
    return dt, 3 * (nx + 1) * (ny + 1) * (nz + 1), v.last_iters


def cpu_matvec_full(dims, E, nu, u=None):
    """One full-size element-by-element K u on the host cores with the oracle's
    restatement of the reference's gather / GEMM / bincount apply
    (core/multigrid.py:318-341), in x-slabs of elements to bound host memory;
    returns (seconds, dof, K u)."""
    from oracle import hex8
    nx, ny, nz = dims
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    KE = hex8.hex8_ke(1.0, nu)
    if u is None:
        u = np.random.default_rng(1).standard_normal(ndof)
    Ee = np.asarray(E, dtype=float).reshape(nx, ny, nz)
    slab = max(1, (1 << 19) // (ny * nz))
    t0 = time.perf_counter()
    y = np.zeros(ndof)
    for x0 in range(0, nx, slab):
        x1 = min(nx, x0 + slab)
        ex, ey, ez = np.meshgrid(np.arange(x0, x1), np.arange(ny), np.arange(nz), indexing="ij")
        edof = np.empty((ex.size, 24), dtype=np.int64)
        for k, (ox, oy, oz) in enumerate(hex8.CORNERS):
            nid = hex8.node_id(ex.ravel() + ox, ey.ravel() + oy, ez.ravel() + oz, nx, ny)
            edof[:, 3 * k:3 * k + 3] = 3 * nid[:, None] + np.arange(3)
        y += hex8.element_apply(u, Ee[x0:x1].ravel(), edof, KE, ndof)
    return time.perf_counter() - t0, ndof, y


def cpu_cores():
    try:
        import threadpoolctl
        info = threadpoolctl.threadpool_info()
        if info:
            return int(max(d.get("num_threads", 1) for d in info))
    except Exception:
        pass
    return os.cpu_count() or 1


def cpu_baseline_record(full=None):
    dt, dof, it = cpu_sample_solve()
    mv = None
    if full is not None:
        mt, mdof, _ = cpu_matvec_full(*full)
        mv = {"seconds_per_apply": mt, "mdof_per_s": mdof / mt / 1e6, "dof": mdof,
              "what": "one full-size FP64 element-by-element K u (gather, 24x24 GEMM, bincount scatter) of "
                      "the bench workload, numpy restatement of the reference's apply, host cores"}
    return {"value": dof / dt / 1e6, "unit": UNIT, "cores": cpu_cores(), "kind": "port", "matvec_full_size": mv,
            "port": PORT_NOTE,
            "sample": (f"numpy restatement of the reference's Jacobi-PCG (core/fea.py:497-593) to {TOL:g} "
                       f"on the seeded bracket generator at {CPU_SAMPLE['shape'][0]}x{CPU_SAMPLE['shape'][1]}x"
                       f"{CPU_SAMPLE['shape'][2]} ({dof} DOF, {it} iterations, {dt:.1f} s); the reference's "
                       f"MG path does not converge on this geometry"),
            "seconds": dt, "iterations": it}


def gpu_same_sample(device, check_every, steps=5):
    """The mixed-precision device solver on the CPU arm's sample (the same
    seeded 64x32x32 bracket to the same tolerance), timed with CUDA events:
    the like-for-like partner of the CPU figure."""
    import torch
    from voxelsim_fea_b200 import generators
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    p = generators.bracket(shape=CPU_SAMPLE["shape"], seed=CPU_SAMPLE["seed"], sigma=CPU_SAMPLE["sigma"],
                           load_n=CPU_SAMPLE["load"], patch=CPU_SAMPLE["patch"])
    nx, ny, nz = p["dims"]
    m = MGSolver(nx, ny, nz, p["fixed_dofs"], nu=p["nu"], max_levels=4,
                 options=SolverOptions.fast(device=device, check_every=check_every))
    E = mg_modulus(p)
    for _ in range(2):
        m.solve(E, p["f"], tol=TOL)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        u = m.solve(E, p["f"], tol=TOL)
    dt = (time.perf_counter() - t0) / steps
    res = {"mdof_per_s": m.ndof / dt / 1e6, "ms_per_solve": dt * 1e3, "iterations": int(m.last_iters),
           "true_resid": float(m.last_info.true_resid), "dof": int(m.ndof),
           "timing": "host clock around MGSolver.solve (host arrays in, displacement out)"}
    m.close()
    return res


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    for _ in range(args.warmup):
        cpu_sample_solve()
    times = []
    dof = it = 0
    for _ in range(args.steps):
        dt, dof, it = cpu_sample_solve()
        times.append(dt)
    ms = 1e3 * float(np.mean(times))
    value = dof / (ms / 1e3) / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": args.workload, "sample": "bracket_64x32x32", "tol": TOL,
                   "method": "Jacobi-PCG (reference fallback path)", "parallelism": "host cores"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cpu_cores(), "kind": "port",
                         "sample": f"bracket generator 64x32x32 ({dof} DOF, {it} iterations) per step",
                         "port": PORT_NOTE},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- batch of parts
def run_batch(args):
    """N independent seeded parts, edges uniform in {32, 48, ..., 128} per
    axis, each its own solver; one step = set-up + solve of all parts in one
    synchronous vf_solve_batch call (parts run concurrently on their own
    streams).  Timed with the host clock around the call, after a device
    synchronisation (the parts' streams have no single device timeline)."""
    import torch
    from voxelsim_fea_b200 import generators
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions, solve_batch
    rng = np.random.default_rng(1234)
    edges = (32, 48, 64, 80, 96, 112, 128)
    parts, solvers = [], []
    for i in range(args.batch):
        sh = tuple(int(rng.choice(edges)) for _ in range(3))
        p = generators.bracket(shape=sh, seed=5000 + i, sigma=3.0, load_n=2000.0, patch=8)
        p["E_mg"] = mg_modulus(p)
        parts.append(p)
        solvers.append(MGSolver(*sh, p["fixed_dofs"], nu=p["nu"], options=SolverOptions.fast(),
                                n_smooth=args.n_smooth))
    ndof = sum(s.ndof for s in solvers)
    E_list = [p["E_mg"] for p in parts]
    F_list = [p["f"] for p in parts]
    mc = args.max_it or None
    for _ in range(args.warmup):
        solve_batch(solvers, E_list, F_list, tol=TOL, max_cg=mc)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        solve_batch(solvers, E_list, F_list, tol=TOL, max_cg=mc)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / args.steps
    worst = max(s.last_info.true_resid for s in solvers)
    if not (worst < TOL):
        raise SystemExit(f"bench: a batch part missed tol={TOL:g} (true residual {worst:.3e})")
    line = {"metric": METRIC, "value": ndof / (ms / 1e3) / 1e6, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": (DTYPE_MIXED if args.mixed_mode == "outer64"
                      else "f32 (FP64 dots, refinement residual, coarsest solve)"),
            "data": "synthetic (seeded generator)",
            "config": {"workload": f"batch{args.batch}_parts_32-128", "dof": ndof, "parts": args.batch,
                       "iterations_max": max(s.last_iters for s in solvers), "timing": "host clock, synchronous call"}}
    print(json.dumps(line), flush=True)
    for s in solvers:
        s.close()
    return 0


# --------------------------------------------------------------------------- other configurations
def other_configs(args, local):
    """One measured solve of each other configuration of the reference's
    benchmark set, after the headline arm (warm-up call, then one timed call,
    host clock around the synchronous API call, tol 1e-8):
      * 192^3 bracket with 16 load cases as one block call;
      * 64 independent parts, edges in {32..128}, in one batch call;
      * the 512x256x256 two-material part (steel / ABS, per-voxel nu), 6 levels."""
    import torch
    from voxelsim_fea_b200 import generators
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions, solve_batch
    opts = dict(device=local, check_every=args.check_every, smoother=args.smoother,
                smoothed_transfers=args.smoothed_transfers, **level_sweeps_kw(args))
    out = {}

    def timed_call(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, r

    # 192^3, k = 16 load cases (generators.load_cases: direction uniform on the
    # sphere, 1-10 kN on a random 8x8 top patch)
    w = WORKLOADS["bracket_192"]
    p = make_problem(w)
    nx, ny, nz = p["dims"]
    F = generators.load_cases(p, 16, seed=w["seed"] + 1)
    m = MGSolver(nx, ny, nz, p["fixed_dofs"], nu=p["nu"], max_levels=w["levels"], options=SolverOptions.fast(**opts))
    E = mg_modulus(p)
    dt, _ = timed_call(lambda: m.solve_block(E, F, tol=TOL, max_cg=args.max_it or None))
    infos = m.last_block_info
    dev_s = max(i.device_ms for i in infos) / 1e3
    out["bracket_192_block16"] = {"seconds": dt, "dof_per_case": m.ndof, "cases": 16,
                                  "mdof_per_s": 16 * m.ndof / dt / 1e6,
                                  "device_solve_seconds": dev_s,
                                  "device_timing": "CUDA events on each case's stream around its solve, the "
                                                   "longest case (the shared set-up excluded)",
                                  "iterations_max": max(i.iters for i in infos),
                                  "true_resid_max": max(i.true_resid for i in infos),
                                  "what": "k = 16 concurrent solves sharing one operator set-up (vf_solve_block)"}
    m.close()
    del F

    # 64 uneven parts in one batch call
    rng = np.random.default_rng(1234)
    edges = (32, 48, 64, 80, 96, 112, 128)
    parts, solvers = [], []
    for i in range(64):
        sh = tuple(int(rng.choice(edges)) for _ in range(3))
        q = generators.bracket(shape=sh, seed=5000 + i, sigma=3.0, load_n=2000.0, patch=8)
        parts.append(q)
        solvers.append(MGSolver(*sh, q["fixed_dofs"], nu=q["nu"], options=SolverOptions.fast(**opts)))
    ndof = sum(sv.ndof for sv in solvers)
    dt, _ = timed_call(lambda: solve_batch(solvers, [mg_modulus(q) for q in parts], [q["f"] for q in parts],
                                           tol=TOL, max_cg=args.max_it or None))
    dev_s = max(sv.last_info.setup_ms + sv.last_info.device_ms for sv in solvers) / 1e3
    out["batch64_parts_32-128"] = {"seconds": dt, "dof": ndof, "mdof_per_s": ndof / dt / 1e6,
                                   "device_part_seconds_max": dev_s,
                                   "device_timing": "CUDA events on each part's stream around its set-up and "
                                                    "solve, the longest part (the parts run concurrently)",
                                   "iterations_max": max(sv.last_iters for sv in solvers),
                                   "true_resid_max": max(sv.last_info.true_resid for sv in solvers),
                                   "what": "independent solvers set up and solved concurrently (vf_solve_batch)"}
    for sv in solvers:
        sv.close()
    del parts, solvers

    # 512 x 256 x 256 two-material part
    w = WORKLOADS["twomat_512x256x256"]
    p = make_problem(w)
    nx, ny, nz = p["dims"]
    m = MGSolver(nx, ny, nz, p["fixed_dofs"], nu=0.3, max_levels=w["levels"], options=SolverOptions.fast(**opts))
    E = mg_modulus(p)
    nu = np.ascontiguousarray(p["nu"], dtype=np.float64)
    cap = args.max_it or 4000
    dt, _ = timed_call(lambda: m.solve(E, p["f"], tol=TOL, max_cg=cap, nu_elem=nu))
    out["twomat_512x256x256"] = {"seconds": dt, "dof": m.ndof, "mdof_per_s": m.ndof / dt / 1e6,
                                 "iterations": int(m.last_iters), "true_resid": float(m.last_info.true_resid),
                                 "converged": bool(m.last_converged), "max_cg": cap,
                                 "setup_ms": float(m.last_info.setup_ms)}
    m.close()
    return out


# --------------------------------------------------------------------------- B200 arm
def run_b200(args):
    import torch
    from voxelsim_fea_b200 import _lib
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    w = WORKLOADS[args.workload]
    p = make_problem(w)
    nx, ny, nz = p["dims"]
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    nelem = nx * ny * nz
    E_mg = mg_modulus(p)
    L = _lib.load()
    DEV = _lib.VF_SOLVE_DEVICE_PTRS

    per_voxel_nu = np.ndim(p["nu"]) > 0
    nu_scalar = 0.3 if per_voxel_nu else float(p["nu"])

    def solver(opts):
        return MGSolver(nx, ny, nz, p["fixed_dofs"], nu=nu_scalar, max_levels=w["levels"], options=opts,
                        n_smooth=args.n_smooth)

    fkw = dict(device=local, check_every=args.check_every, modal_zchunk=args.modal_zchunk, mixed_mode=args.mixed_mode,
               smoother=args.smoother, smoothed_transfers=args.smoothed_transfers, **level_sweeps_kw(args))
    if args.inner_tol is not None:
        fkw["inner_tol"] = args.inner_tol
    fast = solver(SolverOptions.fast(**fkw))
    E_d = torch.from_numpy(np.ascontiguousarray(E_mg)).cuda()
    nu_d = torch.from_numpy(np.ascontiguousarray(p["nu"], dtype=np.float64)).cuda() if per_voxel_nu else None
    nu_ptr = ctypes.c_void_p(nu_d.data_ptr()) if per_voxel_nu else None
    f_d = torch.from_numpy(np.ascontiguousarray(p["f"], dtype=np.float64)).cuda()
    u_d = torch.empty(ndof, dtype=torch.float64, device="cuda")
    info = _lib.VfSolveInfo()
    K = max(1, args.block)
    if K > 1:
        from voxelsim_fea_b200 import generators
        F_d = torch.from_numpy(np.ascontiguousarray(generators.load_cases(p, K, seed=w["seed"] + 1))).cuda()
        U_d = torch.empty_like(F_d)
        infos = (_lib.VfSolveInfo * K)()

    def step(sv):
        _lib.check(L.vf_set_material(sv._h, ctypes.c_void_p(E_d.data_ptr()), nu_ptr, DEV), sv._h)
        if K > 1:
            rc = L.vf_solve_block(sv._h, ctypes.c_void_p(F_d.data_ptr()), K, TOL, args.max_it, DEV,
                                  ctypes.c_void_p(U_d.data_ptr()), infos)
            _lib.check(rc, sv._h)
            return (max(i.iters for i in infos), max(i.true_resid for i in infos),
                    max(i.outer_iters for i in infos))
        rc = L.vf_solve(sv._h, ctypes.c_void_p(f_d.data_ptr()), None, TOL, args.max_it, DEV,
                        ctypes.c_void_p(u_d.data_ptr()), ctypes.byref(info))
        _lib.check(rc, sv._h)
        return info.iters, info.true_resid, info.outer_iters

    stream_ptr = ctypes.c_void_p()
    L.vf_get_stream(fast._h, ctypes.byref(stream_ptr))
    ext = torch.cuda.ExternalStream(stream_ptr.value)

    def timed(sv, steps, warmup, sampler=None):
        for _ in range(warmup):
            step(sv)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        s0 = ctypes.c_uint64()
        L.vf_launch_count(ctypes.byref(s0))
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.start()
        if args.nvtx:
            torch.cuda.nvtx.range_push("vf_timed")
        ev0.record(ext)
        res = None
        for _ in range(steps):
            res = step(sv)
        ev1.record(ext)
        if args.nvtx:
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        if dist:
            dist.barrier()
        s1 = ctypes.c_uint64()
        L.vf_launch_count(ctypes.byref(s1))
        ms = max_over_ranks(ev0.elapsed_time(ev1) / steps, dist, "cuda")
        return ms, res, clocks, int(s1.value - s0.value)

    if args.kernel_profile == "learned":
        # set-up once, then the learned stage (restriction, the 10 U-Net
        # convolutions on level 1, prolongation) once inside NVTX range vf_kernel
        from voxelsim_fea_b200.learned import stage
        step(fast)
        stage.enable_default(fast)
        r = np.random.default_rng(3).standard_normal(ndof)
        e = np.empty(ndof)
        _lib.check(L.vf_learned_apply(fast._h, _lib.ptr(r), _lib.ptr(e)), fast._h)   # warm
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("vf_kernel")
        t0 = time.perf_counter()
        for _ in range(args.kernel_iters):
            _lib.check(L.vf_learned_apply(fast._h, _lib.ptr(r), _lib.ptr(e)), fast._h)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / args.kernel_iters
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"kernel": "learned", "ms_per_application": dt * 1e3, "workload": args.workload,
                          "timing": "host clock around vf_learned_apply (host arrays, FP64 transfers)"}), flush=True)
        fast.close()
        return 0

    if args.kernel_profile:
        # set-up once, then KERNEL alone inside an NVTX range (for ncu --nvtx-include "vf_kernel/")
        kid = {"apply": 0, "smooth": 1, "resid": 2, "restrict": 3, "prolong": 4, "vcycle": 5}[args.kernel_profile]
        prec = _lib.VF_PREC_FP64 if args.kernel_precision == "fp64" else _lib.VF_PREC_FP32
        step(fast)
        torch.cuda.synchronize()
        kms = ctypes.c_double()
        torch.cuda.nvtx.range_push("vf_kernel")
        _lib.check(L.vf_time_kernel(fast._h, kid, prec, args.kernel_iters, ctypes.byref(kms)), fast._h)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"kernel": args.kernel_profile, "precision": args.kernel_precision,
                          "ms_per_launch": kms.value, "workload": args.workload}), flush=True)
        fast.close()
        return 0

    sampler = ClockSampler(local) if rank == 0 else None
    ms, (iters, true_resid, outer), clocks, launches = timed(fast, args.steps, args.warmup, sampler)
    setup_ms = float(info.setup_ms) if K == 1 else None   # set-up part of the last timed step
    if not (true_resid < TOL):
        # a solve that did not reach the tolerance is not a time-to-solution
        raise SystemExit(f"bench: solve did not reach tol={TOL:g} (true residual {true_resid:.3e}, "
                         f"{iters} iterations): no valid measurement")
    value = world * K * ndof / (ms / 1e3) / 1e6
    u_mixed = u_d.cpu().numpy() if K == 1 else None

    # Displacement and von Mises error of every arm against an FP64 solve
    # converged far below the bench tolerance (same geometry, load and
    # hierarchy, FP64 throughout, relative residual < REF_TOL).
    E_stress = np.ascontiguousarray(p["E_stress"], dtype=np.float64)
    nu_host = np.ascontiguousarray(p["nu"], dtype=np.float64) if per_voxel_nu else None
    act_u8 = np.ascontiguousarray(p["active"], dtype=np.uint8)
    node_act = active_nodes(p)
    elem_act = np.asarray(p["active"], dtype=bool)

    def von_mises(u):
        vm = np.empty(nelem)
        _lib.check(L.vf_von_mises(fast._h, _lib.ptr(np.ascontiguousarray(u)), _lib.ptr(E_stress),
                                  _lib.ptr(nu_host), _lib.ptr(act_u8), _lib.ptr(vm)), fast._h)
        return vm

    # plain FP64 GMG-PCG (same hierarchy, FP64 everywhere) on the same GPU
    plain = None
    ref_fields = None
    u_plain = None
    if not args.no_plain or (K == 1 and not args.no_errors):
        ps = solver(SolverOptions.robust(device=local, check_every=args.check_every, smoother=args.smoother,
                                         smoothed_transfers=args.smoothed_transfers, **level_sweeps_kw(args)))
        L.vf_get_stream(ps._h, ctypes.byref(stream_ptr))
        ext_plain = torch.cuda.ExternalStream(stream_ptr.value)
        ext_save = ext
        ext = ext_plain
        if not args.no_plain:
            pms, (pit, pres, _), _, _ = timed(ps, max(1, args.steps // 2), 1)
            plain = {"ms_per_solve": pms, "iterations": pit, "true_resid": pres,
                     "mdof_per_s": ndof / (pms / 1e3) / 1e6, "speedup_of_mixed": pms / ms}
            u_plain = u_d.cpu().numpy() if K == 1 else None
        ext = ext_save
        if K == 1 and not args.no_errors:
            _lib.check(L.vf_set_material(ps._h, ctypes.c_void_p(E_d.data_ptr()), nu_ptr, DEV), ps._h)
            rinfo = _lib.VfSolveInfo()
            rc = L.vf_solve(ps._h, ctypes.c_void_p(f_d.data_ptr()), None, REF_TOL, 20000, DEV,
                            ctypes.c_void_p(u_d.data_ptr()), ctypes.byref(rinfo))
            if rc == _lib.VF_OK and rinfo.true_resid < 1e3 * REF_TOL:
                u_ref = u_d.cpu().numpy()
                ref_fields = (u_ref, von_mises(u_ref), {"tol": REF_TOL, "iterations": int(rinfo.iters),
                                                        "true_resid": float(rinfo.true_resid)})
            else:
                print(f"bench: FP64 reference solve did not converge (status {rc}, true residual "
                      f"{rinfo.true_resid:.3e}); no error figures", file=sys.stderr)
        ps.close()

    def errors_of(u):
        if ref_fields is None or u is None:
            return None
        return field_errors(u, von_mises(u), ref_fields[0], ref_fields[1], node_act, elem_act, apply_k=apply_fp64)

    def apply_fp64(v):
        """K v with the FP64 fine operator (vf_apply, level 0)."""
        y = np.empty(ndof)
        _lib.check(L.vf_apply(fast._h, 0, _lib.VF_PREC_FP64, _lib.ptr(np.ascontiguousarray(v, dtype=np.float64)),
                              _lib.ptr(y)), fast._h)
        return y

    # learned stage + mixed precision (flexible CG with the U-Net stage after
    # each V-cycle), packaged weights; reported beside the mixed solver
    learned = None
    if not args.no_learned:
        from voxelsim_fea_b200.learned import stage
        ls = solver(SolverOptions.fast(**fkw))
        stage.enable_default(ls)
        L.vf_get_stream(ls._h, ctypes.byref(stream_ptr))
        ext_save = ext
        ext = torch.cuda.ExternalStream(stream_ptr.value)
        lms, (lit, lres, lout), _, _ = timed(ls, max(1, args.steps // 2), 1)
        ext = ext_save
        learned = {"ms_per_solve": lms, "iterations": lit, "true_resid": lres, "corrections": lout,
                   "mdof_per_s": ndof / (lms / 1e3) / 1e6,
                   "speedup_vs_plain_fp64": (plain["ms_per_solve"] / lms) if plain else None,
                   "converged": bool(lres < TOL)}
        if K == 1:
            learned["errors_vs_fp64_ref"] = errors_of(u_d.cpu().numpy())
        ls.close()
    if plain is not None:
        plain["errors_vs_fp64_ref"] = errors_of(u_plain)

    # roofline of the dominant kernel: fused FP32 Jacobi sweep on the fine level
    nodes = (nx + 1) * (ny + 1) * (nz + 1)
    kms = ctypes.c_double()
    _lib.check(L.vf_time_kernel(fast._h, 1, _lib.VF_PREC_FP32, 50, ctypes.byref(kms)), fast._h)
    sweep_bytes = 53 * nodes   # u, b, Minv (12 B each), E 4 B, mask 1 B, u' 12 B per node
    amv = ctypes.c_double()
    _lib.check(L.vf_time_kernel(fast._h, 0, _lib.VF_PREC_FP32, 50, ctypes.byref(amv)), fast._h)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = sweep_bytes / (kms.value / 1e3) / 1e9
    traffic, traffic_src = profiled_traffic()
    a64 = ctypes.c_double()
    _lib.check(L.vf_time_kernel(fast._h, 0, _lib.VF_PREC_FP64, 50, ctypes.byref(a64)), fast._h)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "traffic_unit": "B per launch (dram read + write)",
                "traffic_source": traffic_src,
                "kernel": "k_modal_tma<float, SMOOTH> (fused damped-Jacobi sweep, level 0, TMA-staged)",
                "ms_per_launch": kms.value, "algorithmic_bytes_per_launch": sweep_bytes,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst)" if peaks else "fallback 6650 GB/s",
                "matvec_ms_per_launch": amv.value,
                "matvec_gbs": 29 * nodes / (amv.value / 1e3) / 1e9,
                "matvec_frac": 29 * nodes / (amv.value / 1e3) / 1e9 / peak,
                "matvec_fp64_ms_per_launch": a64.value,
                "matvec_fp64_gbs": 57 * nodes / (a64.value / 1e3) / 1e9}

    # e2e through the public API: modulus and load in, displacement out, host
    # numpy arrays in page-locked memory, every step
    e2e = None
    if not args.no_e2e:
        def pinned(a):
            t = torch.empty(np.size(a), dtype=torch.float64, pin_memory=True)
            h = t.numpy()
            h[:] = np.ravel(a)
            return t, h
        f_t, f_h = pinned(p["f"])
        E_t, E_h = pinned(E_mg)
        nu_t, nu_h = pinned(p["nu"]) if per_voxel_nu else (None, None)
        u_t, u_pin = pinned(np.zeros(ndof))
        for _ in range(1):
            fast.solve(E_h, f_h, tol=TOL, max_cg=args.max_it or None, nu_elem=nu_h, out=u_pin)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        ke = max(1, args.steps)
        for _ in range(ke):
            u_h = fast.solve(E_h, f_h, tol=TOL, max_cg=args.max_it or None, nu_elem=nu_h, out=u_pin)
        t1 = time.perf_counter()
        ems = max_over_ranks((t1 - t0) * 1e3 / ke, dist, "cuda")
        e2e = {"value": world * ndof / (ems / 1e3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(8 * nelem + 8 * ndof), "d2h_bytes_per_step": int(8 * ndof),
               "ms_per_step": ems, "true_resid": float(fast.last_info.true_resid),
               "u_finite": bool(np.isfinite(u_h).all())}

    others = None
    if rank == 0 and world == 1 and K == 1 and not args.no_other_configs and args.workload == "bracket_256x128x128":
        others = other_configs(args, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_record(full=((nx, ny, nz), E_mg, nu_scalar))
        same = gpu_same_sample(local, args.check_every)
        same["speedup_vs_cpu"] = same["mdof_per_s"] / cpu["value"]
        cpu["gpu_same_sample"] = same
        if cpu.get("matvec_full_size"):
            mv = cpu["matvec_full_size"]
            mv["device_fp64_ms_per_apply"] = a64.value
            mv["device_fp64_speedup"] = mv["seconds_per_apply"] * 1e3 / a64.value

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": (DTYPE_MIXED if args.mixed_mode == "outer64"
                      else "f32 (FP64 dots, refinement residual, coarsest solve)"),
            "data": "synthetic (seeded generator)",
            "config": {"workload": args.workload + (f"_block{K}" if K > 1 else ""), "dof": ndof,
                       "rhs_per_step": K, "active_voxels": int(p["active"].sum()),
                       "levels": w["levels"], "solver": "mixed-precision GMG-PCG, Galerkin coarse ops, "
                                                        "FP64 Cholesky coarsest", "mixed_mode": args.mixed_mode,
                       "tol": TOL, "l2": "working set > 126 MB L2 (vectors 54-107 MB each)",
                       "parallelism": f"replicas x{world}"},
            "iterations": iters, "outer_iterations": outer, "true_resid": true_resid,
            "errors_vs_fp64_ref": errors_of(u_mixed),
            "fp64_ref": ref_fields[2] if ref_fields else None,
            "setup_ms_per_step": setup_ms,
            "time_to_solution_s": ms / 1e3,
            "plain_fp64": plain,
            "learned_mixed": learned,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "other_configs": others,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    fast.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="bracket_256x128x128")
    ap.add_argument("--check-every", type=int, default=8)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-stage arm")
    ap.add_argument("--max-it", type=int, default=0, help="PCG iteration cap (0: the solver default, 1000)")
    ap.add_argument("--block", type=int, default=1, help="k load cases per step as one block solve")
    ap.add_argument("--n-smooth", type=int, default=2, help="pre/post sweeps of the V-cycle")
    ap.add_argument("--batch", type=int, default=0,
                    help="N independent parts (edges 32..128) per step in one vf_solve_batch call")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-errors", action="store_true", help="skip the FP64 reference solve and the error figures")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the single-solve figures of the 192^3 block, 64-part batch and 512x256x256 configs")
    ap.add_argument("--nvtx", action="store_true", help="wrap the timed steps in NVTX range vf_timed")
    ap.add_argument("--kernel-profile", choices=("apply", "smooth", "resid", "restrict", "prolong", "vcycle", "learned"),
                    help="set up, then run one kernel 3x inside NVTX range vf_kernel and exit")
    ap.add_argument("--kernel-precision", choices=("fp32", "fp64"), default="fp32")
    ap.add_argument("--modal-zchunk", type=int, default=0, help="z-planes per CTA of the modal kernel (0 = auto)")
    ap.add_argument("--kernel-iters", type=int, default=3, help="launches timed by --kernel-profile")
    ap.add_argument("--mixed-mode", choices=("outer64", "reliable", "restart"), default="outer64")
    ap.add_argument("--smoother", choices=("jacobi", "chebyshev"), default="chebyshev",
                    help="V-cycle smoothing of every arm (plain FP64, mixed, learned)")
    ap.add_argument("--smoothed-transfers", type=int, default=2,
                    help="bitmask of transfers l -> l+1 with the smoothed prolongation (2: level 1 -> 2)")
    ap.add_argument("--smoothed-level-sweeps", type=int, default=None,
                    help="sweeps on the level above a smoothed transfer (default: the presets' choice)")
    ap.add_argument("--inner-tol", type=float, default=None,
                    help="mixed: residual reduction between FP64 corrections (solver default if unset)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.batch:
        return run_batch(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
