"""Level operators on the device vs the reference's own outputs (golden vectors
from core/multigrid.py on a 16x8x8 grid with lognormal E, x=0 face clamped)
and vs the sparse Galerkin oracle.  Calls go through the C-ABI (MGSolver's
private-API mirrors route to vf_apply / vf_smooth / ...)."""

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

FP32_RTOL = 2e-6   # relative to the max |entry| of the FP64 reference result


def _solver(g, **opt):
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    nx, ny, nz = (int(v) for v in g["dims"])
    m = MGSolver(nx, ny, nz, g["fixed"], nu=float(g["nu"]), options=SolverOptions(**opt))
    m.set_density(g["E"])
    return m


def _close(a, ref, rtol):
    scale = np.abs(ref).max()
    err = np.abs(a - ref).max()
    assert err <= rtol * scale, f"max err {err:.3e} vs scale {scale:.3e}"


@pytest.mark.parametrize("prec,rtol", [("fp64", 1e-13), ("fp32", FP32_RTOL)])
def test_apply_every_level(gpu, prec, rtol):
    g = golden("mg_ops_16x8x8.npz")
    m = _solver(g)
    assert len(m.levels) == int(g["n_levels"])
    for li in range(len(m.levels)):
        _close(m._apply(li, g[f"u{li}"], precision=prec), g[f"Ku{li}"], rtol)


def test_inverse_diagonal(gpu):
    g = golden("mg_ops_16x8x8.npz")
    m = _solver(g)
    for li in range(len(m.levels)):
        np.testing.assert_allclose(m.inv_diagonal(li), g[f"Minv{li}"], rtol=1e-14)
        np.testing.assert_array_equal(m.levels[li]["free"], g[f"free{li}"])


@pytest.mark.parametrize("prec,rtol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_smooth_restrict_prolong(gpu, prec, rtol):
    g = golden("mg_ops_16x8x8.npz")
    m = _solver(g)
    for li in range(len(m.levels)):
        u0 = g[f"u{li}"] * g[f"free{li}"]
        _close(m._smooth(li, u0, g[f"b{li}"], 2, precision=prec), g[f"smooth{li}"], rtol)
        if li + 1 < len(m.levels):
            _close(m._restrict(li, g[f"u{li}"], precision=prec), g[f"restrict{li}"], rtol)
            _close(m._prolongate(li, g[f"ec{li}"], precision=prec), g[f"prolong{li}"], rtol)


@pytest.mark.parametrize("prec,rtol", [("fp64", 1e-11), ("fp32", 1e-4)])
def test_vcycle(gpu, prec, rtol):
    g = golden("mg_ops_16x8x8.npz")
    m = _solver(g)
    _close(m._vcycle(0, g["vc_r"], precision=prec), g["vc_z"], rtol)


# FP16 storage of the scaled stencil: ~5e-4 relative per entry (2^-11),
# summed over 27 blocks
HALF_STENCIL_RTOL = 3e-3


@pytest.mark.parametrize("storage", ["sym_half", "sym", "full"])
def test_galerkin_levels_match_sparse_rap(gpu, storage):
    """Device Galerkin stencils (built from the matrix-free fine level, then
    stencil RAP) act like the scipy R A P hierarchy on every level, in every
    storage format (symmetric scaled FP16 / FP32 / FP64, or full)."""
    from oracle import galerkin
    g = golden("mg_ops_16x8x8.npz")
    nx, ny, nz = (int(v) for v in g["dims"])
    m = _solver(g, coarse="galerkin", coarse_storage=storage)
    hier = galerkin.galerkin_hierarchy(nx, ny, nz, g["E"], g["fixed"], nu=float(g["nu"]))
    rng = np.random.default_rng(5)
    for li, (A, free) in enumerate(hier):
        u = rng.standard_normal(A.shape[0])
        ref = A @ (u * free) if li > 0 else A @ u
        ref = ref * free
        _close(m._apply(li, u * free, precision="fp64"), ref, 1e-12)
        tol32 = HALF_STENCIL_RTOL if (storage == "sym_half" and li > 0) else FP32_RTOL
        _close(m._apply(li, u * free, precision="fp32"), ref, tol32)


def test_galerkin_with_interior_dirichlet_and_lame(gpu):
    """Masked general path of the level-1 build (Dirichlet DOFs inside the
    grid, single components) with a per-voxel Poisson ratio."""
    from oracle import galerkin, hex8
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    rng = np.random.default_rng(11)
    nx, ny, nz = 8, 8, 4
    ne = nx * ny * nz
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    E = np.exp(rng.normal(0, 1, ne))
    nu = np.where(rng.random(ne) < 0.5, 0.3, 0.35)
    fixed = np.unique(rng.choice(ndof, 60, replace=False))
    lam, mu = hex8.lame(E, nu)
    hier = galerkin.galerkin_hierarchy(nx, ny, nz, None, fixed, lam=lam, mu=mu, max_levels=3)
    m = MGSolver(nx, ny, nz, fixed, nu=0.3, max_levels=3, options=SolverOptions(coarse="galerkin"))
    m.set_density(E, nu_elem=nu)
    for li, (A, free) in enumerate(hier):
        u = rng.standard_normal(A.shape[0]) * free
        _close(m._apply(li, u), (A @ u) * free, 1e-12)


def test_lame_fine_operator(gpu):
    """Per-voxel Poisson ratio: Ke = lam K_lam + mu K_mu on the fine level."""
    from oracle import hex8
    from voxelsim_fea_b200.multigrid import MGSolver
    rng = np.random.default_rng(3)
    nx, ny, nz = 6, 5, 4
    ne = nx * ny * nz
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    E = np.exp(rng.normal(0, 1, ne))
    nu = rng.uniform(0.2, 0.4, ne)
    m = MGSolver(nx, ny, nz, np.zeros(0, np.int64), nu=0.3)
    m.set_density(E, nu_elem=nu)
    u = rng.standard_normal(ndof)
    lam, mu = hex8.lame(E, nu)
    ref = hex8.element_apply_lame(u, lam, mu, hex8.build_edof(nx, ny, nz), ndof)
    _close(m._apply(0, u), ref, 1e-13)
    _close(m._apply(0, u, precision="fp32"), ref, FP32_RTOL)


def test_operator_is_deterministic(gpu):
    g = golden("mg_ops_16x8x8.npz")
    m = _solver(g)
    a = m._vcycle(0, g["vc_r"])
    b = m._vcycle(0, g["vc_r"])
    assert np.array_equal(a, b)
