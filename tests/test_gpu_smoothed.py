"""The coarse space with a smoothed prolongation on the transfer from level 1
to level 2 (vf_options.smoothed_transfers = 2), against the host restatement
oracle.galerkin.smoothed_hierarchy given the device's own lambda_1:

* the reach-2 (125-block) level-2 operator and the level-3 operator below it
  (trilinear transfer from a reach-2 level), FP64 to 1e-11, FP32 with FP16
  scaled storage to 3e-3 of the result scale; the coarse free masks;
* the smoothed restriction P_s^T r and prolongation P_s e between levels 1
  and 2;
* solves: FP64 and mixed precision reach the tolerance (true FP64 residual),
  in fewer iterations than the trilinear hierarchy, with the same
  displacement, on a two-material part with a per-voxel Poisson ratio.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _part(shape=(32, 16, 16), seed=3):
    from voxelsim_fea_b200.learned.train import make_part
    return make_part(seed, shape=shape)


def _solver(part, smoothed, fast=False, **kw):
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    nx, ny, nz = part["dims"]
    preset = SolverOptions.fast if fast else SolverOptions.robust
    return MGSolver(nx, ny, nz, part["fixed"], nu=0.3,
                    options=preset(smoothed_transfers=2 if smoothed else 0, **kw))


@pytest.fixture(scope="module")
def hierarchy(gpu):
    from oracle import galerkin, hex8
    part = _part()
    nx, ny, nz = part["dims"]
    m = _solver(part, True)
    m.set_density(part["E"], nu_elem=part["nu"])
    assert len(m.levels) == 4
    lam1 = m.level_omega(1)[1]
    lam_e, mu_e = hex8.lame(part["E"], part["nu"])
    levels, Ps = galerkin.smoothed_hierarchy(nx, ny, nz, None, part["fixed"], lam=lam_e, mu=mu_e,
                                             smoothed={1}, lams={1: lam1})
    yield m, levels, Ps
    m.close()


@pytest.mark.parametrize("li", [2, 3])
def test_wide_level_operator(hierarchy, li):
    from voxelsim_fea_b200 import _lib
    m, levels, _ = hierarchy
    A, free = levels[li]
    rng = np.random.default_rng(li)
    u = rng.standard_normal(A.shape[0])
    ref = A @ u
    scale = np.abs(ref).max()
    y = m._apply(li, u)
    assert np.abs(y - ref).max() <= 1e-11 * scale
    y32 = m._apply(li, u, precision="fp32")
    assert np.abs(y32 - ref).max() <= 3e-3 * scale
    out = np.empty(A.shape[0] // 3, dtype=np.uint8)
    _lib.check(_lib.load().vf_level_mask(m._h, li, out.ctypes.data_as(ctypes.c_void_p)), m._h)
    bits = ((out[:, None] >> np.arange(3)) & 1).astype(bool).ravel()
    np.testing.assert_array_equal(bits, free)


def test_smoothed_transfers(hierarchy):
    m, levels, Ps = hierarchy
    P = Ps[1]                      # level 1 -> 2
    rng = np.random.default_rng(11)
    r = rng.standard_normal(P.shape[0])
    ref_r = P.T @ (r * levels[1][1])
    rc = m._restrict(1, r)
    assert np.abs(rc - ref_r).max() <= 1e-12 * np.abs(ref_r).max()
    e = rng.standard_normal(P.shape[1]) * levels[2][1]
    ref_e = P @ e
    ef = m._prolongate(1, e)
    assert np.abs(ef - ref_e).max() <= 1e-12 * np.abs(ref_e).max()


@pytest.mark.parametrize("fast", [False, True])
def test_smoothed_solve(gpu, fast):
    part = _part(shape=(48, 48, 48), seed=9_015_838)
    res = {}
    for smoothed in (False, True):
        m = _solver(part, smoothed, fast=fast)
        u = m.solve(part["E"], part["f"], tol=1e-8, nu_elem=part["nu"], max_cg=3000)
        res[smoothed] = (u, m.last_iters, m.last_converged, m.last_info.true_resid)
        m.close()
    (u0, it0, c0, _), (u1, it1, c1, r1) = res[False], res[True]
    assert c0 and c1 and r1 < 1e-8
    assert it1 < it0, (it1, it0)
    assert np.abs(u1 - u0).max() <= 1e-5 * np.abs(u0).max()


@pytest.mark.parametrize("fast", [False, True])
def test_smoothed_level_sweeps(gpu, fast):
    """One sweep before and after the coarse correction on level 1, whose
    smoothed restriction and prolongation smooth it once each already: the
    same displacement in about as many iterations as two sweeps."""
    part = _part(shape=(48, 48, 48), seed=9_015_838)
    res = {}
    for sw in (0, 1):
        m = _solver(part, True, fast=fast, smoothed_level_sweeps=sw)
        u = m.solve(part["E"], part["f"], tol=1e-8, nu_elem=part["nu"], max_cg=3000)
        res[sw] = (u, m.last_iters, m.last_converged, m.last_info.true_resid)
        m.close()
    (u0, it0, c0, _), (u1, it1, c1, r1) = res[0], res[1]
    assert c0 and c1 and r1 < 1e-8
    assert it1 <= int(1.15 * it0) + 3, (it1, it0)
    assert np.abs(u1 - u0).max() <= 1e-5 * np.abs(u0).max()
