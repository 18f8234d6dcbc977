"""Independent parts of uneven size set up and solved in one call give the
same displacements as one solve per part."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_equals_separate_solves(gpu):
    from voxelsim_fea_b200 import generators
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions, solve_batch
    shapes = [(32, 48, 32), (64, 32, 48), (48, 48, 64), (32, 32, 32), (80, 48, 32)]
    parts, solvers = [], []
    for i, sh in enumerate(shapes):
        p = generators.bracket(shape=sh, seed=100 + i, sigma=3.0, load_n=2000.0, patch=8)
        p["E_mg"] = np.where(p["active"], p["E_stiff"], p["E_stiff"] * 1e-9)
        parts.append(p)
        solvers.append(MGSolver(*sh, p["fixed_dofs"], nu=p["nu"], options=SolverOptions.fast()))
    U = solve_batch(solvers, [p["E_mg"] for p in parts], [p["f"] for p in parts], tol=1e-8)
    for s, p, u in zip(solvers, parts, U):
        assert s.last_converged and s.last_info.true_resid < 1e-8
        ref = s.solve(p["E_mg"], p["f"], tol=1e-8)
        np.testing.assert_array_equal(u, ref)
