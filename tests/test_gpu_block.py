"""Block right-hand sides: k load cases on one geometry in one call give the
same displacements as k separate solves (the reference's one-call-per-case
path), for the mixed and the FP64 solver, and across a change of material."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem():
    from voxelsim_fea_b200 import generators
    p = generators.bracket(shape=(64, 32, 32), seed=3, sigma=4.0, load_n=5000.0, patch=16)
    E = np.where(p["active"], p["E_stiff"], p["E_stiff"] * 1e-9)
    F = generators.load_cases(p, 4, seed=11)
    return p, E, F


@pytest.mark.parametrize("preset", ["fast", "robust"])
def test_block_equals_separate_solves(gpu, preset):
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    p, E, F = _problem()
    nx, ny, nz = p["dims"]
    opts = getattr(SolverOptions, preset)()
    m = MGSolver(nx, ny, nz, p["fixed_dofs"], nu=p["nu"], max_levels=4, options=opts)
    U = m.solve_block(E, F, tol=1e-8)
    assert m.last_converged
    assert all(i.true_resid < 1e-8 for i in m.last_block_info)
    for j in range(F.shape[0]):
        u = m.solve(E, F[j], tol=1e-8)
        np.testing.assert_array_equal(U[j], u)   # same kernels, same operator, deterministic


def test_block_after_material_change(gpu):
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    p, E, F = _problem()
    nx, ny, nz = p["dims"]
    m = MGSolver(nx, ny, nz, p["fixed_dofs"], nu=p["nu"], max_levels=4, options=SolverOptions.fast())
    m.solve_block(E, F[:2], tol=1e-8)
    E2 = E * np.where(np.arange(E.size) % 3 == 0, 2.0, 1.0)
    U = m.solve_block(E2, F[:3], tol=1e-8)
    for j in range(3):
        u = m.solve(E2, F[j], tol=1e-8)
        np.testing.assert_array_equal(U[j], u)
