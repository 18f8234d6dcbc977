"""libvoxfea loads and exports every symbol include/voxfea.h declares; host-only
entry points work without a GPU (no device compute is called here)."""

import ctypes
import os
import re

import numpy as np

from conftest import REPO, golden


def _declared_symbols():
    text = open(os.path.join(REPO, "include", "voxfea.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(vf_[a-z0-9_]+)\s*\(", text))
    names.discard("vf_progress_fn")
    return names


def test_exports_match_header(lib):
    from voxelsim_fea_b200 import _lib
    declared = _declared_symbols()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in voxfea.h but not exported"
    assert declared == set(_lib.EXPORTS)


def test_abi_and_options(lib):
    from voxelsim_fea_b200 import _lib
    assert lib.vf_abi_version() == 1
    o = _lib.default_options()
    assert o.struct_size == ctypes.sizeof(_lib.VfOptions)
    assert (o.n_smooth, o.min_elems, o.max_levels, o.coarse_sweeps) == (2, 4, 6, 30)
    assert abs(o.omega - 0.6) < 1e-15
    assert o.mixed_mode == _lib.MIXED_MODES["outer64"] and o.modal_zchunk == 0 and o.autotune == 1
    assert o.smoother == _lib.SMOOTHERS["jacobi"] and o.cheb_ratio == 30
    assert lib.vf_status_string(_lib.VF_ERR_STALLED) == b"MG-PCG stalled/diverged"


def test_host_hex8_tables_match_reference(lib):
    """The C++ restatement of _hex8_KE / _hex8_B_C (host code of the library)."""
    g = golden("hex8.npz")
    for nu in (0.30, 0.33, 0.35):
        KE = np.empty(576)
        KL = np.empty(576)
        KM = np.empty(576)
        B0 = np.empty(144)
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        assert lib.vf_hex8_tables(nu, p(KE), p(KL), p(KM), p(B0)) == 0
        tag = int(round(nu * 100))
        np.testing.assert_allclose(KE.reshape(24, 24), g[f"KE_{tag}"], atol=2e-16)
        np.testing.assert_allclose(B0.reshape(6, 24), g[f"B0_{tag}"], atol=0)
        lam = nu / ((1 + nu) * (1 - 2 * nu))
        mu = 1 / (2 * (1 + nu))
        np.testing.assert_allclose(lam * KL + mu * KM, KE, atol=1e-15)
    assert lib.vf_hex8_tables(0.5, None, None, None, None) == 1


def test_create_rejects_bad_args(lib):
    from voxelsim_fea_b200 import _lib
    h = ctypes.c_void_p()
    assert lib.vf_create(0, 4, 4, 0.3, None, ctypes.byref(h)) == _lib.VF_ERR_ARG
    assert lib.vf_create(4, 4, 4, 0.7, None, ctypes.byref(h)) == _lib.VF_ERR_ARG
    o = _lib.default_options()
    o.struct_size = 3
    assert lib.vf_create(4, 4, 4, 0.3, ctypes.byref(o), ctypes.byref(h)) == _lib.VF_ERR_ARG
    # option fields outside their enums are refused before any device call
    for field, bad in (("mixed_mode", 3), ("mixed_mode", -1), ("modal_zchunk", -2), ("fine_kernel", 3),
                       ("coarse_storage", 3), ("precision", 3)):
        o = _lib.default_options()
        setattr(o, field, bad)
        assert lib.vf_create(4, 4, 4, 0.3, ctypes.byref(o), ctypes.byref(h)) == _lib.VF_ERR_ARG, field
    # Chebyshev smoothing needs the lambda estimates, at most 2 sweeps and kernels that take its step
    for fields in ({}, {"omega_mode": 1, "n_smooth": 3}, {"omega_mode": 1, "smoothed_level_sweeps": 3},
                   {"omega_mode": 1, "fine_kernel": 1},
                   {"omega_mode": 1, "coarse_storage": 2}, {"omega_mode": 1, "cheb_ratio": 1}):
        o = _lib.default_options()
        o.smoother = _lib.SMOOTHERS["chebyshev"]
        for k, v in fields.items():
            setattr(o, k, v)
        assert lib.vf_create(4, 4, 4, 0.3, ctypes.byref(o), ctypes.byref(h)) == _lib.VF_ERR_ARG, fields
    assert not h.value


def test_grid_assembly_matches_reference_semantics():
    """The oracle's restatement of the grid assembly (the checker of the
    device assembly, vf_assemble_grid) on role masks: active = build &
    ~exclude, fixed DOFs per bearing axis flags, load split evenly over the
    load nodes (solve_worker.py:242-270)."""
    from oracle.assemble import assemble
    dims = (2, 1, 1)
    nn = 3 * 2 * 2
    build = np.array([True, True])
    excl = np.array([False, True])
    bearing = np.zeros(nn, dtype=bool)
    bearing[[0, 3]] = True
    load = np.zeros(nn, dtype=bool)
    load[[2, 5, 11]] = True
    descr = [("build", None), ("exclude", None), ("bearing", (True, False, True)), ("load", (3.0, 0.0, -6.0))]
    active, fixed, f = assemble(descr, [build, excl, bearing, load], dims)
    np.testing.assert_array_equal(active, [True, False])
    np.testing.assert_array_equal(fixed, [0, 2, 9, 11])
    assert f[3 * 2] == 1.0 and f[3 * 5 + 2] == -2.0 and f[3 * 11] == 1.0 and abs(f.sum() - (-3.0)) < 1e-15


def test_presets_pick_a_supported_smoother():
    """robust() / fast() smooth with Chebyshev polynomials unless the chosen
    kernels or damping cannot take its step; the reference preset keeps Jacobi."""
    from voxelsim_fea_b200.multigrid import SolverOptions
    assert SolverOptions().smoother == "jacobi"
    assert SolverOptions.reference().smoother == "jacobi"
    assert SolverOptions.robust().smoother == "chebyshev"
    assert SolverOptions.fast().smoother == "chebyshev"
    assert SolverOptions.robust(fine_kernel="gather").smoother == "jacobi"
    assert SolverOptions.fast(coarse_storage="full").smoother == "jacobi"
    assert SolverOptions.robust(omega_mode="fixed").smoother == "jacobi"
    assert SolverOptions.robust(smoother="jacobi").smoother == "jacobi"
    # one smoothing step on level 1 above the smoothed level 1 -> 2 transfer
    assert SolverOptions.robust().smoothed_level_sweeps == 1 and SolverOptions.fast().smoothed_level_sweeps == 1
    assert SolverOptions.fast(smoothed_transfers=0).smoothed_level_sweeps == 0
    assert SolverOptions().smoothed_level_sweeps == 0
