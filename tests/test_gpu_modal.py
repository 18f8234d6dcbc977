"""The modal z-marching fine operator (default kernel, TMA-staged; and its
cp.async-staged form) against the CPU oracle
and against the 27-neighbour gather kernel, on odd-sized grids that exercise
partial tiles in x/y and unequal z-lanes, for several z-chunk sizes, both
epilogues that carry extra data (Jacobi sweep, residual), FP64 and FP32, and a
per-voxel Poisson ratio."""

import numpy as np
import pytest

from oracle import hex8

pytestmark = pytest.mark.gpu

RTOL = {"fp64": 1e-13, "fp32": 2e-6}


def _close(a, ref, rtol):
    scale = np.abs(ref).max()
    err = np.abs(a - ref).max()
    assert err <= rtol * scale, f"max err {err:.3e} vs scale {scale:.3e}"


def _problem(nx, ny, nz, seed, lame=False):
    rng = np.random.default_rng(seed)
    ne = nx * ny * nz
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    E = np.exp(rng.normal(0.0, 1.5, ne))
    E[rng.random(ne) < 0.3] *= 1e-6            # void-like contrast
    fixed = np.unique(rng.choice(ndof, ndof // 20, replace=False))
    nu = rng.uniform(0.25, 0.4, ne) if lame else None
    return rng, E, fixed, nu, ndof


@pytest.mark.parametrize("zchunk", [-1, 0, 1, 2, 5, 64])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_modal_apply_matches_oracle(gpu, zchunk, prec):
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    nx, ny, nz = 37, 23, 19
    rng, E, fixed, _, ndof = _problem(nx, ny, nz, 7)
    m = MGSolver(nx, ny, nz, fixed, nu=0.31, options=SolverOptions(modal_zchunk=zchunk))
    m.set_density(E)
    free = m.levels[0]["free"]
    u = rng.standard_normal(ndof)
    ref = hex8.element_apply(u, E, hex8.build_edof(nx, ny, nz), hex8.hex8_ke(1.0, 0.31), ndof) * free
    _close(m._apply(0, u, precision=prec), ref, RTOL[prec])


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_modal_smooth_and_lame_match_gather(gpu, prec):
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    nx, ny, nz = 34, 31, 9
    rng, E, fixed, nu, ndof = _problem(nx, ny, nz, 11, lame=True)
    a = MGSolver(nx, ny, nz, fixed, nu=0.3, options=SolverOptions(fine_kernel="modal", modal_zchunk=3))
    b = MGSolver(nx, ny, nz, fixed, nu=0.3, options=SolverOptions(fine_kernel="gather"))
    c = MGSolver(nx, ny, nz, fixed, nu=0.3, options=SolverOptions(fine_kernel="modal_cpasync", modal_zchunk=5))
    for m in (a, b, c):
        m.set_density(E, nu_elem=nu)
    free = a.levels[0]["free"]
    u = rng.standard_normal(ndof) * free
    rhs = rng.standard_normal(ndof) * free
    lam, mu = hex8.lame(E, nu)
    ref = hex8.element_apply_lame(u, lam, mu, hex8.build_edof(nx, ny, nz), ndof) * free
    _close(a._apply(0, u, precision=prec), ref, RTOL[prec])
    _close(a._apply(0, u, precision=prec), b._apply(0, u, precision=prec), RTOL[prec])
    _close(a._smooth(0, u, rhs, 3, precision=prec), b._smooth(0, u, rhs, 3, precision=prec),
           10 * RTOL[prec])
    # the TMA-staged and the cp.async-staged forms do identical arithmetic
    np.testing.assert_array_equal(a._apply(0, u, precision=prec), c._apply(0, u, precision=prec))
    np.testing.assert_array_equal(a._smooth(0, u, rhs, 3, precision=prec), c._smooth(0, u, rhs, 3, precision=prec))


def test_modal_solve_matches_gather_solve(gpu):
    """Same solution and (to rounding) the same iteration count with either
    kernel (both with Jacobi smoothing, the one the gather kernel supports)."""
    from voxelsim_fea_b200 import generators
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    p = generators.bracket(shape=(64, 32, 32), seed=0, sigma=4.0, load_n=5000.0, patch=16)
    nx, ny, nz = p["dims"]
    E_mg = np.where(p["active"], p["E_stiff"], p["E_stiff"] * 1e-9)
    out = {}
    for k in ("modal", "gather"):
        m = MGSolver(nx, ny, nz, p["fixed_dofs"], nu=p["nu"], max_levels=4,
                     options=SolverOptions.robust(fine_kernel=k, smoother="jacobi"))
        out[k] = (m.solve(E_mg, p["f"], tol=1e-9), m.last_iters)
    ua, ia = out["modal"]
    ub, ib = out["gather"]
    assert abs(ia - ib) <= 2
    assert np.abs(ua - ub).max() < 1e-7 * np.abs(ub).max()


@pytest.mark.parametrize("dims", [(64, 48, 40), (120, 60, 50), (200, 13, 3)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_modal_even_wave_is_bitwise_chunked(gpu, dims, prec):
    """The one-wave split (z-chunk -1: CTAs share the (tile, plane) units
    evenly, a range crossing a tile boundary marched as a second segment, the
    staging ring carried across segments) does each node's arithmetic exactly
    as the per-chunk grid does: bitwise equal apply and Jacobi sweeps, with a
    per-voxel Poisson ratio, on grids with several units per CTA."""
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    nx, ny, nz = dims
    rng, E, fixed, nu, ndof = _problem(nx, ny, nz, 5, lame=True)
    ms = {}
    for zc in (-1, 3):
        ms[zc] = MGSolver(nx, ny, nz, fixed, nu=0.3, max_levels=1,
                          options=SolverOptions(fine_kernel="modal", modal_zchunk=zc, autotune=False))
        ms[zc].set_density(E, nu_elem=nu)
    free = ms[3].levels[0]["free"]
    u = rng.standard_normal(ndof) * free
    rhs = rng.standard_normal(ndof) * free
    a, b = ms[-1], ms[3]
    np.testing.assert_array_equal(a._apply(0, u, precision=prec), b._apply(0, u, precision=prec))
    np.testing.assert_array_equal(a._smooth(0, u, rhs, 2, precision=prec), b._smooth(0, u, rhs, 2, precision=prec))
    if prec == "fp64":
        lam, mu = hex8.lame(E, nu)
        ref = hex8.element_apply_lame(u, lam, mu, hex8.build_edof(nx, ny, nz), ndof) * free
        _close(a._apply(0, u, precision=prec), ref, RTOL[prec])
