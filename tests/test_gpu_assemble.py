"""Grid assembly of a solve job on the device (vf_assemble_grid, the
reference worker's core/solve_worker.py:242-270) against its numpy
restatement (oracle.assemble): several build masks (the last one wins),
overlapping exclusions, bearings fixing different axes, loads that overlap,
one load that reaches no node -- active set, fixed DOFs and the force vector
bit for bit; and the island pre-step from the fixed-DOF bits against the
oracle's flood fill (core/fea.py:207-227)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _job(seed, dims):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    ne, nn = nx * ny * nz, (nx + 1) * (ny + 1) * (nz + 1)
    descr, masks = [], []
    descr.append(("build", None)); masks.append(rng.random(ne) < 0.3)
    descr.append(("load", (10.0, -3.0, 7.5))); masks.append(rng.random(nn) < 0.05)
    descr.append(("build", None)); masks.append(rng.random(ne) < 0.8)
    descr.append(("exclude", None)); masks.append(rng.random(ne) < 0.1)
    descr.append(("bearing", (True, False, True))); masks.append(rng.random(nn) < 0.05)
    descr.append(("load", (0.0, 0.0, -1000.0))); masks.append(rng.random(nn) < 0.02)
    descr.append(("exclude", None)); masks.append(rng.random(ne) < 0.1)
    descr.append(("bearing", (False, True, False))); masks.append(rng.random(nn) < 0.05)
    descr.append(("load", (1.0, 2.0, 3.0))); masks.append(np.zeros(nn, dtype=bool))
    return descr, masks


@pytest.mark.parametrize("dims", [(9, 7, 5), (40, 24, 16)])
def test_assembly_matches_restatement(gpu, dims):
    from oracle.assemble import assemble as ref_assemble
    from voxelsim_fea_b200.solve_worker import assemble
    descr, masks = _job(5, dims)
    a0, f0, F0 = ref_assemble(descr, masks, dims)
    a1, f1, F1, bits = assemble(descr, masks, dims)
    np.testing.assert_array_equal(a1, a0)
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(F1, F0)          # same divisions, same order of sums
    assert bits.shape == ((dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1),)


def test_islands_from_bits(gpu):
    from oracle import islands
    from voxelsim_fea_b200.solve_worker import assemble, drop_unsupported_islands_bits
    dims = (20, 12, 10)
    descr, masks = _job(8, dims)
    active, fixed, _, bits = assemble(descr, masks, dims)
    kept_ref, nrem_ref = islands.drop_unsupported_islands(active.reshape(dims), fixed)
    kept, nrem = drop_unsupported_islands_bits(active, bits, dims)
    assert nrem == nrem_ref
    np.testing.assert_array_equal(kept, np.asarray(kept_ref).ravel())
