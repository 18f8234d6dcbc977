"""The job wire format end to end: the reference's job.pkl (a box part with an
exclusion, a bearing box, a load box; tests/golden/make_golden.py) through
this package's worker gives the reference worker's final.pkl -- the same keys,
identical voxel masks and island count; with the job's ``solver`` set to
"reference" (the reference's multigrid algorithm) the same CG iteration count
and stress / displacement / safety fields to 1e-5; with the default robust
hierarchy (fewer iterations) the same fields to the solver tolerance."""

import importlib.util
import os
import pickle

import numpy as np
import pytest

from conftest import REPO, golden

pytestmark = pytest.mark.gpu


def _job(solver="reference"):
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(REPO, "tests", "golden",
                                                                            "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    job = mg._worker_job()
    if solver:
        job["solver"] = solver
    return job


def _check(final, ref, same_solver=True):
    assert set(ref.keys()) <= set(final.keys())
    np.testing.assert_array_equal(final["active3d"], ref["active3d"])
    assert final["n_islands_removed"] == int(ref["n_islands_removed"])
    assert final["cg_converged"]
    if same_solver:
        assert final["cg_iters"] == int(ref["cg_iters"])
        np.testing.assert_allclose(final["cg_resid_history"], ref["cg_resid_history"], rtol=1e-6)
    else:
        assert final["cg_iters"] <= int(ref["cg_iters"])
    tol = 1e-5 if same_solver else 1e-3
    for k in ("stress3d", "displacement3d", "safety3d"):
        a, b = np.asarray(final[k], dtype=float), np.asarray(ref[k], dtype=float)
        assert np.abs(a - b).max() <= tol * np.abs(b).max(), k
    for k in ("max_stress_pa", "stress_vmax", "max_displacement_m", "min_safety_factor", "displacement_vmax_m"):
        assert abs(float(final[k]) - float(ref[k])) <= tol * abs(float(ref[k])), k
    assert final["reliable"] == bool(ref["reliable"])


def test_worker_matches_reference_final(gpu, tmp_path):
    from voxelsim_fea_b200 import solve_worker
    jp = tmp_path / "job.pkl"
    with open(jp, "wb") as fh:
        pickle.dump(_job(), fh)
    solve_worker._worker_main(str(jp), str(tmp_path))
    with open(tmp_path / "status.json") as fh:
        assert fh.read().count('"done"') == 1
    with open(tmp_path / "final.pkl", "rb") as fh:
        final = pickle.load(fh)
    _check(final, dict(golden("worker_28x10x8.npz")))


def test_solver_client_round_trip(gpu):
    """The reference's job dict unchanged (default robust hierarchy), through
    the subprocess client."""
    from voxelsim_fea_b200.solve_worker import SolverClient
    c = SolverClient()
    c.start(_job(solver=None))
    try:
        ev, final = c.wait(timeout=300)
        assert ev == "done", final
        _check(final, dict(golden("worker_28x10x8.npz")), same_solver=False)
    finally:
        c.cleanup()


def test_worker_reports_missing_supports(gpu, tmp_path):
    from voxelsim_fea_b200 import solve_worker
    job = _job()
    job["descr"][2] = ("bearing", (False, False, False))
    jp = tmp_path / "job.pkl"
    with open(jp, "wb") as fh:
        pickle.dump(job, fh)
    solve_worker._worker_main(str(jp), str(tmp_path))
    import json
    with open(tmp_path / "status.json") as fh:
        st = json.load(fh)
    assert st["phase"] == "error" and "No supports" in st["error"]
