"""The learned preconditioner stage inside the solver: the C++ inference
path equals the training-side forward (torch glue + the same conv kernels),
flexible CG equals PCG for a fixed preconditioner, a solve with the stage
converges to the same solution, and the trained network's correction removes
more A-norm error per application than an untrained network's."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (48, 48, 48)


def _part(seed):
    from voxelsim_fea_b200.learned import train
    return train.make_part(seed, shape=SHAPE)


def test_inference_matches_training_forward(gpu):
    import torch
    from voxelsim_fea_b200.learned import stage, train, unet
    part = _part(123)
    p = train.make_pairs(part, 1, (4,))[0]
    net = unet.UNet(7).cuda()
    with torch.no_grad():
        for w in net.w:
            w.mul_(3.0)
    ef_t = train.predict_fine(net, p).detach().cpu().numpy().reshape(-1)
    m = train.solver_for(part)
    m.set_density(part["E"], nu_elem=part["nu"])
    stage.configure(m, net.flat_params(), 1, False)
    ef_c = stage.apply(m, m._apply(0, p.e.cpu().numpy().reshape(-1).astype(float)))
    # BF16 activations: agreement to the BF16 rounding of ~10 layers
    assert np.abs(ef_c - ef_t).max() < 3e-2 * np.abs(ef_t).max()


def test_flexible_cg_equals_pcg_for_fixed_preconditioner(gpu):
    from voxelsim_fea_b200 import generators
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    c = generators.cantilever()
    out = {}
    for flex in (False, True):
        m = MGSolver(*c["dims"], c["fixed_dofs"], nu=c["nu"], options=SolverOptions.robust(flexible=flex))
        out[flex] = (m.solve(c["E_stiff"], c["f"], tol=1e-10), m.last_iters)
    assert out[True][1] == out[False][1]
    assert np.abs(out[True][0] - out[False][0]).max() < 1e-8 * np.abs(out[False][0]).max()


def test_solve_with_learned_stage_converges(gpu):
    from voxelsim_fea_b200.learned import stage
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    part = _part(4242)
    nx, ny, nz = part["dims"]
    sols = {}
    for use in (False, True):
        m = MGSolver(nx, ny, nz, part["fixed"], nu=0.3, options=SolverOptions.robust())
        m.set_density(part["E"], nu_elem=part["nu"])
        if use:
            stage.enable_default(m)
        sols[use] = m.solve(part["E"], part["f"], tol=1e-8, nu_elem=part["nu"])
        assert m.last_converged and m.last_info.true_resid < 1e-8
    ref = sols[False]
    assert np.abs(sols[True] - ref).max() < 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("fast", [False, True])
def test_learned_stage_falls_back_to_plain_pcg(gpu, fast):
    """With the stage on, a residual that stops halving over learned_watch
    iterations switches the stage off and the solve goes on as plain PCG from
    its current iterate (FP64 PCG and the FP64-outer / FP32-V-cycle mode): a
    tiny watch window forces the switch early; the solve converges to the
    plain solve's displacement and reports the switch iteration."""
    from voxelsim_fea_b200.learned import stage
    from voxelsim_fea_b200.multigrid import MGSolver, SolverOptions
    part = _part(4242)
    nx, ny, nz = part["dims"]
    preset = SolverOptions.fast if fast else SolverOptions.robust
    res = {}
    for watch, use in ((64, False), (1, True), (0, True)):
        m = MGSolver(nx, ny, nz, part["fixed"], nu=0.3, options=preset(learned_watch=watch))
        m.set_density(part["E"], nu_elem=part["nu"])
        if use:
            stage.enable_default(m)
        u = m.solve(part["E"], part["f"], tol=1e-8, nu_elem=part["nu"])
        res[(watch, use)] = (u, m.last_converged, m.last_info.true_resid, int(m.last_info.outer_iters),
                             m.last_iters)
        m.close()
    ref = res[(64, False)][0]
    u, conv, tr, switched, iters = res[(1, True)]
    assert conv and tr < 1e-8
    assert 0 < switched < iters, (switched, iters)
    assert np.abs(u - ref).max() < 1e-5 * np.abs(ref).max()
    assert res[(0, True)][3] == 0          # watch off: the stage stays on to the end
    assert res[(64, False)][3] == 0


def _energy_left(m, c, e, r):
    """A-norm error fraction after the optimal step along c: 1 - cos_A^2(c, e)."""
    Ac = m._apply(0, c)
    cr = float(c @ r)
    return 1.0 - cr * cr / (float(c @ Ac) * float(e @ r))


def test_trained_network_gain_per_application(gpu):
    """On held-out parts (seeds disjoint from training) the trained network's
    correction removes more of the V-cycle iteration's slow error (in the A
    norm, at the optimal step the solver takes) than an untrained network."""
    from voxelsim_fea_b200.learned import stage, train, unet
    params, level = stage.load_weights()
    fresh = unet.UNet(11).flat_params()
    left = {"trained": [], "untrained": []}
    for seed in (9_100_003, 9_200_003):
        part = _part(seed)
        p = train.make_pairs(part, level, (8,))[0]
        m = train.solver_for(part)
        m.set_density(part["E"], nu_elem=part["nu"])
        e = p.e.cpu().numpy().reshape(-1).astype(float)
        r = m._apply(0, e)
        for name, w in (("trained", params), ("untrained", fresh)):
            stage.configure(m, w, level, False)
            left[name].append(_energy_left(m, stage.apply(m, r), e, r))
    print("A-norm error left after one stage application:", left)
    assert np.mean(left["trained"]) < np.mean(left["untrained"])
