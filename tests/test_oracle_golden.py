"""The CPU oracle reproduces the reference's own outputs (golden vectors made
by tests/golden/make_golden.py from core/fea.py and core/multigrid.py)."""

import numpy as np
import pytest

from conftest import golden
from oracle import fea as ofea
from oracle import hex8, islands, mg


@pytest.mark.parametrize("nu", [0.30, 0.33, 0.35])
def test_hex8_tables(nu):
    g = golden("hex8.npz")
    tag = int(round(nu * 100))
    np.testing.assert_allclose(hex8.hex8_ke(1.0, nu), g[f"KE_{tag}"], rtol=0, atol=1e-15)
    B, C = hex8.hex8_b_c(nu)
    np.testing.assert_allclose(B, g[f"B0_{tag}"], atol=1e-15)
    np.testing.assert_allclose(C, g[f"C0_{tag}"], atol=1e-15)
    lam, mu = hex8.lame(1.0, nu)
    KL, KM = hex8.lame_split()
    np.testing.assert_allclose(lam * KL + mu * KM, g[f"KE_{tag}"], atol=1e-14)


def test_edof():
    np.testing.assert_array_equal(hex8.build_edof(3, 2, 4), golden("hex8.npz")["edof_3x2x4"])


def test_level_operators():
    g = golden("mg_ops_16x8x8.npz")
    nx, ny, nz = (int(v) for v in g["dims"])
    m = mg.MGOracle(nx, ny, nz, g["fixed"], nu=float(g["nu"]))
    m.set_density(g["E"])
    assert len(m.levels) == int(g["n_levels"])
    for li in range(len(m.levels)):
        np.testing.assert_array_equal(m.levels[li]["free"], g[f"free{li}"])
        np.testing.assert_allclose(m.levels[li]["Minv"], g[f"Minv{li}"], rtol=1e-14)
        np.testing.assert_allclose(m.apply(li, g[f"u{li}"]), g[f"Ku{li}"], rtol=1e-12, atol=1e-12)
        u0 = g[f"u{li}"] * g[f"free{li}"]
        np.testing.assert_allclose(m.smooth(li, u0, g[f"b{li}"], 2), g[f"smooth{li}"],
                                   rtol=1e-12, atol=1e-12)
        if li + 1 < len(m.levels):
            np.testing.assert_allclose(m.restrict(li, g[f"u{li}"]), g[f"restrict{li}"], atol=1e-12)
            np.testing.assert_allclose(m.prolongate(li, g[f"ec{li}"]), g[f"prolong{li}"], atol=1e-12)
    np.testing.assert_allclose(m.vcycle(0, g["vc_r"]), g["vc_z"], rtol=1e-11, atol=1e-12)


def test_cantilever_solve_pins_reference():
    g = golden("cantilever_64x16x16_L3.npz")
    from voxelsim_fea_b200 import generators
    p = generators.cantilever()
    m = mg.MGOracle(*p["dims"], p["fixed_dofs"], nu=p["nu"], max_levels=3)
    u = m.solve(p["E_stiff"], p["f"], tol=1e-8)
    assert m.last_iters == int(g["iters"]) == 19
    np.testing.assert_allclose(m.resid_history, g["resid_history"], rtol=1e-6, atol=1e-14)
    np.testing.assert_allclose(u, g["u"], rtol=0, atol=1e-10 * np.abs(g["u"]).max())
    # known answers of the cantilever (tip deflection ~ -8.22e-5 m, max VM ~ 91.66 MPa)
    assert abs(u[2::3].min() / -8.36e-5 - 1) < 0.05
    assert abs(g["vm"].max() / 91.66e6 - 1) < 1e-3


def test_noise_jacobi_pins_reference():
    g = golden("noise_32x16x16_jacobi.npz")
    nx, ny, nz = (int(v) for v in g["dims"])
    v = ofea.VoxelFEAOracle(nx, ny, nz, nu=float(g["nu"]), active_elems=g["active"],
                            use_multigrid=False)
    v.set_fixed(g["fixed"])
    u = v.solve(g["E_stiff"], g["f"], tol=1e-10)
    assert v.last_iters == int(g["iters"])
    np.testing.assert_allclose(u, g["u"], atol=1e-12 * np.abs(g["u"]).max())
    vm = v.element_von_mises_stress(u, g["E_stress"]) / float(g["vsize"])
    np.testing.assert_allclose(vm, g["vm"], rtol=1e-9, atol=1e-6 * g["vm"].max())
    np.testing.assert_allclose(v.element_strain_energy(u), g["se"], rtol=1e-9,
                               atol=1e-12 * g["se"].max())


def test_islands():
    g = golden("islands_12x10x8.npz")
    nx, ny, nz = g["active"].shape
    np.testing.assert_array_equal(islands.seed_from_fixed_dofs(nx, ny, nz, g["fixed"]), g["seed"])
    kept, n = islands.drop_unsupported_islands(g["active"], g["fixed"])
    np.testing.assert_array_equal(kept, g["kept"])
    assert n == int(g["n_removed"])


def test_galerkin_oracle_equals_rediscretization_for_uniform_E():
    """Sanity of the sparse RAP oracle: with uniform E and no Dirichlet DOFs,
    Galerkin coarsening of Q1 hex8 equals rediscretization (x 2 per level)."""
    from oracle import galerkin
    nx, ny, nz = 8, 4, 4
    E = np.full(nx * ny * nz, 3.0)
    hier = galerkin.galerkin_hierarchy(nx, ny, nz, E, np.zeros(0, np.int64), max_levels=2)
    A1 = hier[1][0]
    K1 = galerkin.fine_matrix(4, 2, 2, np.full(16, 3.0 * 2.0))
    assert abs(A1 - K1).max() < 1e-12 * abs(K1).max()


def test_voxelize_oracle_matches_reference():
    """oracle/voxelize.py against the reference's own parity ray cast
    (inside_worker._inside_mask_numpy, voxel_centers, node_coords)."""
    from oracle import voxelize
    g = golden("inside_cases.npz")
    dims, origin, vsize = tuple(int(v) for v in g["dims"]), g["origin"], float(g["vsize"])
    np.testing.assert_array_equal(voxelize.voxel_centers(dims, origin, vsize), g["centers"])
    np.testing.assert_array_equal(voxelize.node_coords(dims, origin, vsize), g["nodes"])
    np.testing.assert_array_equal(voxelize.RAY_DIR, g["ray_dir"])
    for name in ("box", "torus", "tilted"):
        v, f = g[f"{name}_verts"], g[f"{name}_faces"]
        for key, pts in (("points", g[f"{name}_points"]), ("centers", g["centers"]), ("nodes", g["nodes"])):
            np.testing.assert_array_equal(voxelize.inside_mask(v, f, pts), g[f"{name}_in_{key}"], err_msg=f"{name}/{key}")


def test_bench_cpu_matvec_slabs_match_oracle_apply():
    """The CPU baseline's full-size K u (bench.py, x-slabs of elements) is the
    oracle's element apply, on a grid that takes several slabs."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(os.path.dirname(__file__), "..", "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    from oracle import hex8
    nx, ny, nz = 40, 30, 500
    rng = np.random.default_rng(0)
    E = rng.random(nx * ny * nz)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    u = rng.standard_normal(ndof)
    _, dof, y = bench.cpu_matvec_full((nx, ny, nz), E, 0.3, u=u)
    yr = hex8.element_apply(u, E, hex8.build_edof(nx, ny, nz), hex8.hex8_ke(1.0, 0.3), ndof)
    assert dof == ndof
    assert np.abs(y - yr).max() <= 1e-14 * np.abs(yr).max()


def _mg_pcg(levels, Ps, f, tol=1e-8, maxit=500):
    """Galerkin MG-PCG on host sparse levels: Jacobi V(2,2) (omega = 1.6 /
    padded lambda_max), dense coarsest solve; returns the iteration count."""
    from oracle.galerkin import _lambda_max
    info = []
    for A, free in levels:
        d = A.diagonal()
        dinv = np.where(free & (d > 0), 1.0 / np.where(d > 0, d, 1.0), 0.0)
        info.append((A, free, dinv, 1.6 / (1.1 * _lambda_max(A, dinv, free))))
    Ac = levels[-1][0].toarray()
    fc = levels[-1][1]
    Ac[~fc, ~fc] = 1.0
    Acinv = np.linalg.inv(Ac)

    def vc(i, b):
        A, free, dinv, w = info[i]
        if i == len(info) - 1:
            return (Acinv @ b) * free
        x = w * dinv * b
        x = x + w * dinv * (b - A @ x)
        x = x + Ps[i] @ vc(i + 1, Ps[i].T @ (b - A @ x))
        for _ in range(2):
            x = x + w * dinv * (b - A @ x)
        return x

    A = info[0][0]
    x = np.zeros_like(f)
    r = f.copy()
    z = vc(0, r)
    p = z.copy()
    rz = r @ z
    for it in range(1, maxit + 1):
        Ap = A @ p
        a = rz / (p @ Ap)
        x += a * p
        r -= a * Ap
        if np.linalg.norm(r) < tol * np.linalg.norm(f):
            return it
        z = vc(0, r)
        rz, rz_old = r @ z, rz
        p = z + (rz / rz_old) * p
    return maxit


def test_smoothed_prolongation_hierarchy():
    """The smoothed-prolongation Galerkin levels: symmetric coarse operators,
    P_l = D (P - omega/lambda D^-1 A P), coarse stencils two nodes wide, and
    fewer MG-PCG iterations than the trilinear Galerkin hierarchy on a
    voided lognormal-modulus part."""
    from oracle import galerkin
    nx, ny, nz = 16, 16, 8
    rng = np.random.default_rng(11)
    E = np.exp(rng.normal(0.0, 1.0, nx * ny * nz))
    E[rng.random(E.size) < 0.3] *= 1e-6
    fixed = np.arange(3 * (nx + 1) * (ny + 1))                 # z = 0 face
    levels, Ps = galerkin.smoothed_hierarchy(nx, ny, nz, E, fixed, max_levels=3)
    plain = galerkin.galerkin_hierarchy(nx, ny, nz, E, fixed, max_levels=3)
    for A, _ in levels:
        assert abs(A - A.T).max() <= 1e-12 * abs(A).max()
    # the level-1 operator couples nodes two apart (125 blocks) where the trilinear one stops at one
    nnz_s, nnz_t = levels[1][0].nnz, plain[1][0].nnz
    assert nnz_s > 3 * nnz_t
    f = np.zeros(levels[0][0].shape[0])
    f[-3 * (nx + 1) * (ny + 1) + 2::3] = -1.0
    f *= levels[0][1]
    from oracle.mg import level_dims
    dims = level_dims(nx, ny, nz, 4, 3)
    Pt = [galerkin.prolong_matrix(dims[i], dims[i + 1]) for i in range(len(dims) - 1)]
    Pt = [sp_mask(P, plain[i][1], plain[i + 1][1]) for i, P in enumerate(Pt)]
    it_s = _mg_pcg(levels, Ps, f)
    it_t = _mg_pcg(plain, Pt, f)
    assert it_s < it_t, (it_s, it_t)


def sp_mask(P, free_f, free_c):
    import scipy.sparse as sp
    return (sp.diags(free_f.astype(float)) @ P @ sp.diags(free_c.astype(float))).tocsr()
