"""Chebyshev smoothing (SolverOptions(smoother="chebyshev")): one V-cycle on a
two-level Galerkin hierarchy against a host restatement with the device's own
lambda estimate and inverse diagonal; the V-cycle as a symmetric operator (PCG
needs one); degree 1 equal to damped Jacobi with the matching weight; solves
to the reference's displacement, with no more iterations than Jacobi on the
noise bracket."""

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _ops(max_levels, **opt):
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    g = golden("mg_ops_16x8x8.npz")
    nx, ny, nz = (int(v) for v in g["dims"])
    m = MGSolver(nx, ny, nz, g["fixed"], nu=float(g["nu"]), max_levels=max_levels,
                 options=SolverOptions.robust(**opt))
    m.set_density(g["E"])
    return g, m


def test_vcycle_matches_host_restatement(gpu):
    from oracle import galerkin
    g, m = _ops(2, smoother="chebyshev")
    nx, ny, nz = (int(v) for v in g["dims"])
    (A0, f0), (Ac, fc) = galerkin.galerkin_hierarchy(nx, ny, nz, g["E"], g["fixed"], nu=float(g["nu"]),
                                                     max_levels=2)
    P = galerkin.prolong_matrix((nx, ny, nz), (nx // 2, ny // 2, nz // 2))
    dinv = m.inv_diagonal(0) * f0
    beta = m.level_omega(0)[1]
    ratio = 30.0
    alpha = beta / ratio
    theta, delta = 0.5 * (beta + alpha), 0.5 * (beta - alpha)
    sigma = theta / delta
    rho0 = 1.0 / sigma
    rho1 = 1.0 / (2.0 * sigma - rho0)
    c2_0, c1_1, c2_1 = 1.0 / theta, rho1 * rho0, 2.0 * rho1 / delta
    Acd = Ac.toarray()
    Acd[~fc, ~fc] = 1.0
    Acinv = np.linalg.inv(Acd)
    r = np.random.default_rng(7).standard_normal(A0.shape[0]) * f0
    # pre-smoothing from zero: x1 = Minv r / theta, x2 = x1 + c1 x1 + c2 Minv (r - A x1)
    x1 = c2_0 * dinv * r
    x = x1 + c1_1 * x1 + c2_1 * dinv * (r - A0 @ x1)
    rc = fc * (P.T @ (r - A0 @ x))
    x = x + f0 * (P @ (Acinv @ rc))
    # post-smoothing: d1 = Minv (r - A x) / theta, x1 = x + d1, x2 = x1 + c1 d1 + c2 Minv (r - A x1)
    d1 = c2_0 * dinv * (r - A0 @ x)
    x1 = x + d1
    ref = x1 + c1_1 * d1 + c2_1 * dinv * (r - A0 @ x1)
    z = m._vcycle(0, r)
    assert np.abs(z - ref).max() <= 1e-10 * np.abs(ref).max()
    m.close()


@pytest.mark.parametrize("smoother", ["jacobi", "chebyshev"])
def test_vcycle_is_symmetric(gpu, smoother):
    g, m = _ops(6, smoother=smoother)
    rng = np.random.default_rng(3)
    free = m.levels[0]["free"]
    r1 = rng.standard_normal(m.ndof) * free
    r2 = rng.standard_normal(m.ndof) * free
    a, b = r2 @ m._vcycle(0, r1), r1 @ m._vcycle(0, r2)
    assert abs(a - b) <= 1e-10 * max(abs(a), abs(b))
    m.close()


def test_degree_one_is_weighted_jacobi(gpu):
    """Degree 1 on [beta / r, beta] is the Jacobi sweep weighted 1/theta =
    (r / (r + 1)) 2 / beta: the Jacobi V(1,1) with omega_rel = r / (r + 1)."""
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    g = golden("mg_ops_16x8x8.npz")
    nx, ny, nz = (int(v) for v in g["dims"])
    a = MGSolver(nx, ny, nz, g["fixed"], nu=float(g["nu"]), n_smooth=1,
                 options=SolverOptions.robust(smoother="chebyshev", cheb_ratio=30))
    b = MGSolver(nx, ny, nz, g["fixed"], nu=float(g["nu"]), n_smooth=1,
                 options=SolverOptions.robust(omega_rel=30.0 / 31.0))
    for m in (a, b):
        m.set_density(g["E"])
    r = np.random.default_rng(1).standard_normal(a.ndof) * a.levels[0]["free"]
    za, zb = a._vcycle(0, r), b._vcycle(0, r)
    assert np.abs(za - zb).max() <= 1e-12 * np.abs(zb).max()
    a.close()
    b.close()


@pytest.mark.parametrize("preset", ["robust", "fast"])
def test_chebyshev_solves(gpu, preset):
    from oracle.fea import true_residual
    from voxelsim_fea_b200 import generators
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    mk = SolverOptions.robust if preset == "robust" else SolverOptions.fast
    # cantilever: the reference's displacement
    gc = golden("cantilever_64x16x16_L3.npz")
    p = generators.cantilever()
    m = MGSolver(*p["dims"], p["fixed_dofs"], nu=p["nu"], options=mk(smoother="chebyshev"))
    u = m.solve(p["E_stiff"], p["f"], tol=1e-10)
    assert m.last_converged and m.last_info.true_resid < 1e-10
    assert np.abs(u - gc["u"]).max() <= 1e-7 * np.abs(gc["u"]).max()
    m.close()
    # noise bracket: converged, true FP64 residual below tol, no more iterations than Jacobi
    p = generators.bracket(shape=(64, 32, 32), seed=0, sigma=4.0, load_n=5000.0, patch=16)
    nx, ny, nz = p["dims"]
    E_mg = np.where(p["active"], p["E_stiff"], p["E_stiff"] * 1e-9)
    its = {}
    for sm in ("jacobi", "chebyshev"):
        m = MGSolver(nx, ny, nz, p["fixed_dofs"], nu=p["nu"], max_levels=4, options=mk(smoother=sm))
        u = m.solve(E_mg, p["f"], tol=1e-8)
        assert m.last_converged
        its[sm] = m.last_iters
        if sm == "chebyshev":
            assert true_residual(nx, ny, nz, E_mg, p["fixed_dofs"], p["f"], u, nu=p["nu"]) < 1e-8
        m.close()
    assert its["chebyshev"] <= its["jacobi"], its
