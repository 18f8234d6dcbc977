"""Generate golden vectors from the reference's own solver code.

Run once in a container where the reference checkout is readable:

    python tests/golden/make_golden.py [--ref /root/reference]

It imports VoxelSim-FEA's ``core.fea`` / ``core.multigrid`` read-only (CPU,
numpy, FP64) and writes small ``.npz`` fixtures next to this script.  The
fixtures pin the CPU oracle (``oracle/``) and, through it, the CUDA path.
Nothing at test time reads the reference checkout.
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _import_reference(ref):
    sys.path.insert(0, ref)
    from core import compute_plan, fea, multigrid  # noqa: F401
    return fea, multigrid


def _mg_ops_case(fea, multigrid):
    """Level operators of the reference MGSolver on a 16x8x8 grid with
    lognormal E, x=0 face clamped (3 levels)."""
    rng = np.random.default_rng(1234)
    nx, ny, nz = 16, 8, 8
    nelem = nx * ny * nz
    E = np.exp(rng.normal(0.0, 1.0, nelem))
    face0 = np.array([0 + (nx + 1) * (iy + (ny + 1) * iz)
                      for iz in range(nz + 1) for iy in range(ny + 1)])
    fixed = np.sort(np.concatenate([3 * face0 + c for c in range(3)]))
    mg = multigrid.MGSolver(nx, ny, nz, fixed, nu=0.3, compute_mode="CPU", xp=np)
    mg.set_density(E)
    out = {"dims": np.array([nx, ny, nz]), "E": E, "fixed": fixed, "nu": 0.3,
           "n_levels": len(mg.levels)}
    for li, lv in enumerate(mg.levels):
        u = rng.standard_normal(lv["ndof"])
        b = rng.standard_normal(lv["ndof"]) * lv["free"]
        out[f"u{li}"] = u
        out[f"b{li}"] = b
        out[f"Ku{li}"] = mg._apply(li, u)
        out[f"Minv{li}"] = np.asarray(lv["Minv"])
        out[f"free{li}"] = np.asarray(lv["free"])
        out[f"smooth{li}"] = mg._smooth(li, u * lv["free"], b, 2)
        if li + 1 < len(mg.levels):
            out[f"restrict{li}"] = mg._restrict(li, u)
            ec = rng.standard_normal(mg.levels[li + 1]["ndof"])
            out[f"ec{li}"] = ec
            out[f"prolong{li}"] = mg._prolongate(li, ec)
    r = rng.standard_normal(mg.levels[0]["ndof"]) * mg.levels[0]["free"]
    out["vc_r"] = r
    out["vc_z"] = mg._vcycle(0, r)
    return out


def _cantilever_case(fea, multigrid, max_levels):
    from voxelsim_fea_b200 import generators
    p = generators.cantilever()
    nx, ny, nz = p["dims"]
    mg = multigrid.MGSolver(nx, ny, nz, p["fixed_dofs"], nu=p["nu"],
                            compute_mode="CPU", max_levels=max_levels)
    u = mg.solve(p["E_stiff"], p["f"], tol=1e-8)
    v = fea.VoxelFEA(nx, ny, nz, nu=p["nu"], compute_mode="CPU")
    vm = v.element_von_mises_stress(u, p["E_stress"]) / p["vsize"]
    return {"u": u, "iters": mg.last_iters, "resid_history": np.array(mg.resid_history),
            "n_levels": len(mg.levels), "vm": vm}


def _noise_case(fea, multigrid):
    """Seeded 32x16x16 noise part (the bracket generator scaled down),
    reference Jacobi-PCG on the active-restricted system to 1e-10."""
    from voxelsim_fea_b200 import generators
    p = generators.bracket(shape=(32, 16, 16), seed=3, sigma=2.0, load_n=500.0, patch=8)
    nx, ny, nz = p["dims"]
    active3d = p["active"].reshape(nx, ny, nz)
    kept, n_removed = fea.drop_unsupported_islands(active3d, p["fixed_dofs"])
    v = fea.VoxelFEA(nx, ny, nz, nu=p["nu"], active_elems=kept, compute_mode="CPU",
                     use_multigrid=False)
    v.set_fixed(p["fixed_dofs"])
    u = v.solve(p["E_stiff"], p["f"], tol=1e-10)
    vm = v.element_von_mises_stress(u, p["E_stress"]) / p["vsize"]
    se = v.element_strain_energy(u)
    return {"active": kept.ravel(), "n_removed": n_removed, "fixed": p["fixed_dofs"],
            "f": p["f"], "E_stiff": p["E_stiff"], "E_stress": p["E_stress"],
            "nu": p["nu"], "vsize": p["vsize"], "dims": np.array([nx, ny, nz]),
            "u": u, "iters": v.last_iters, "vm": vm, "se": se}


def _islands_case(fea):
    rng = np.random.default_rng(77)
    nx, ny, nz = 12, 10, 8
    active = rng.random((nx, ny, nz)) < 0.55
    iy, iz = np.meshgrid(np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    face0 = (0 + (nx + 1) * (iy + (ny + 1) * iz)).ravel()
    fixed = np.sort(np.concatenate([3 * face0, 3 * face0 + 2]))
    seed = fea.seed_from_fixed_dofs(nx, ny, nz, fixed)
    kept, n_removed = fea.drop_unsupported_islands(active, fixed)
    return {"active": active, "fixed": fixed, "seed": seed, "kept": kept,
            "n_removed": n_removed}


def box_mesh(lo, hi):
    """Closed triangulated axis-aligned box (12 outward triangles)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], dtype=float)
    f = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [1, 2, 6], [1, 6, 5], [2, 3, 7], [2, 7, 6], [3, 0, 4], [3, 4, 7]], dtype=np.int64)
    return v, f


def torus_mesh(R, r, nu_, nv_, center):
    """Closed triangulated torus around z (a part with a through-hole)."""
    a = np.linspace(0, 2 * np.pi, nu_, endpoint=False)
    b = np.linspace(0, 2 * np.pi, nv_, endpoint=False)
    A, B = np.meshgrid(a, b, indexing="ij")
    v = np.stack([(R + r * np.cos(B)) * np.cos(A), (R + r * np.cos(B)) * np.sin(A), r * np.sin(B)], -1).reshape(-1, 3)
    v = v + np.asarray(center, dtype=float)
    f = []
    for i in range(nu_):
        for j in range(nv_):
            p, q = i * nv_ + j, ((i + 1) % nu_) * nv_ + j
            p2, q2 = i * nv_ + (j + 1) % nv_, ((i + 1) % nu_) * nv_ + (j + 1) % nv_
            f += [[p, q, q2], [p, q2, p2]]
    return v, np.asarray(f, dtype=np.int64)


def _inside_case(ref):
    """Voxelization: the reference's parity ray cast on three closed meshes,
    for random points, voxel centers and grid nodes (inside_worker.py)."""
    from core import inside_worker as iw
    rng = np.random.default_rng(31)
    out = {}
    meshes = {"box": box_mesh((0.013, 0.021, 0.017), (0.91, 0.57, 0.43)),
              "torus": torus_mesh(0.31, 0.11, 24, 12, (0.5, 0.5, 0.25)),
              "tilted": None}
    v, f = box_mesh((0.1, 0.1, 0.1), (0.7, 0.5, 0.4))
    th = 0.37
    rot = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1.0]])
    meshes["tilted"] = (v @ rot.T + np.array([0.2, 0.05, 0.03]), f)
    dims, origin, vsize = (23, 17, 11), np.array([-0.031, -0.017, -0.009]), 0.047
    centers = iw.voxel_centers(dims, origin, vsize)
    nodes = iw.node_coords(dims, origin, vsize)
    for name, (v, f) in meshes.items():
        pts = rng.uniform(-0.1, 1.1, size=(3000, 3))
        out[f"{name}_verts"] = v
        out[f"{name}_faces"] = f
        out[f"{name}_points"] = pts
        out[f"{name}_in_points"] = iw._inside_mask_numpy(v, f, pts)
        out[f"{name}_in_centers"] = iw._inside_mask_numpy(v, f, centers)
        out[f"{name}_in_nodes"] = iw._inside_mask_numpy(v, f, nodes)
    out["dims"] = np.array(dims)
    out["origin"] = origin
    out["vsize"] = np.array(vsize)
    out["centers"] = centers
    out["nodes"] = nodes
    out["ray_dir"] = iw._RAY_DIR
    return out


def _worker_job():
    """A complete solve job in the reference's job.pkl format: a 28x10x8 grid,
    a box part with a box exclusion, a bearing box at x = 0 clamping x/y/z, a
    load box at x = max with 1 kN in -z."""
    vsize = 0.002
    dims = (28, 10, 8)
    origin = np.array([0.0, 0.0, 0.0])
    part = box_mesh((0.0005, 0.0005, 0.0005), (0.0555, 0.0195, 0.0155))
    excl = box_mesh((0.020, -0.01, 0.009), (0.030, 0.03, 0.02))
    bearing = box_mesh((-0.001, -0.001, -0.001), (0.0015, 0.021, 0.017))
    load = box_mesh((0.0545, -0.001, -0.001), (0.0575, 0.021, 0.017))
    qs = [(part, "centers"), (excl, "centers"), (bearing, "nodes"), (load, "nodes")]
    return {"grid": {"dims": dims, "origin": origin, "vsize": vsize}, "direction": None,
            "queries": [{"verts": v, "faces": f, "target": t} for (v, f), t in qs],
            "descr": [("build", None), ("exclude", None), ("bearing", (True, True, True)),
                      ("load", (0.0, 0.0, -1000.0))],
            "material": {"youngs_modulus": 200e9, "poisson": 0.3, "yield_strength": 250e6},
            "compute_mode": "CPU"}


def _worker_case(ref):
    """The reference worker end to end (job.pkl -> final.pkl)."""
    import pickle
    import tempfile
    from core import solve_worker
    job = _worker_job()
    with tempfile.TemporaryDirectory() as d:
        jp = os.path.join(d, "job.pkl")
        with open(jp, "wb") as fh:
            pickle.dump(job, fh)
        solve_worker._worker_main(jp, d)
        with open(os.path.join(d, "final.pkl"), "rb") as fh:
            final = pickle.load(fh)
    keep = {}
    for k, v in final.items():
        if v is None or isinstance(v, str):
            continue
        keep[k] = np.asarray(v)
    return keep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, REPO)
    fea, multigrid = _import_reference(args.ref)

    ke = {}
    for nu in (0.3, 0.33, 0.35):
        ke[f"KE_{int(round(nu * 100))}"] = fea._hex8_KE(1.0, nu)
        B, C = fea._hex8_B_C(nu)
        ke[f"B0_{int(round(nu * 100))}"] = B
        ke[f"C0_{int(round(nu * 100))}"] = C
    ke["edof_3x2x4"] = fea.build_edof(3, 2, 4)
    np.savez_compressed(os.path.join(HERE, "hex8.npz"), **ke)

    np.savez_compressed(os.path.join(HERE, "mg_ops_16x8x8.npz"), **_mg_ops_case(fea, multigrid))
    c3 = _cantilever_case(fea, multigrid, max_levels=3)
    np.savez_compressed(os.path.join(HERE, "cantilever_64x16x16_L3.npz"), **c3)
    c6 = _cantilever_case(fea, multigrid, max_levels=6)
    np.savez_compressed(os.path.join(HERE, "cantilever_64x16x16_L6.npz"),
                        iters=c6["iters"], resid_history=c6["resid_history"],
                        n_levels=c6["n_levels"], u_tip=c6["u"][2::3].min())
    np.savez_compressed(os.path.join(HERE, "noise_32x16x16_jacobi.npz"), **_noise_case(fea, multigrid))
    np.savez_compressed(os.path.join(HERE, "islands_12x10x8.npz"), **_islands_case(fea))
    np.savez_compressed(os.path.join(HERE, "inside_cases.npz"), **_inside_case(args.ref))
    np.savez_compressed(os.path.join(HERE, "worker_28x10x8.npz"), **_worker_case(args.ref))
    print("cantilever L3 iters", c3["iters"], "L6 iters", c6["iters"],
          "max vm", c3["vm"].max())


if __name__ == "__main__":
    main()
