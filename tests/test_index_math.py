"""Index arithmetic of the modal TMA kernel's work split, restated on the host
(voxelsim_fea_b200/csrc/vf_modal_tma.cu: the (tile, plane) unit ranges of
the per-chunk grid and of the one-wave split, the segments a range crosses,
and the two z-lanes of a segment): every output plane of every tile is
written by exactly one (CTA, lane, step), for grids with partial tiles,
ranges that cross tile boundaries, and more CTAs than units."""

import itertools
import os

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

TX, TY, L = 32, 8, 2   # CTA tile (threads) and z-lanes of the FP32 kernel


def _ranges(lx, ly, lz, zchunk, nb_wave):
    ntx, nty = (lx + TX - 1) // (TX - 1), (ly + TY - 1) // (TY - 1)
    NP = lz + 1
    U = ntx * nty * NP
    if zchunk > 0:
        ntile = ntx * nty
        nb = ntile * ((NP + zchunk - 1) // zchunk)
        for b in range(nb):
            tile, ch = b % ntile, b // ntile
            yield tile * NP + ch * zchunk, tile * NP + min((ch + 1) * zchunk, NP)
    else:
        nb = min(nb_wave, U)
        for b in range(nb):
            yield U * b // nb, U * (b + 1) // nb


def _outputs(lx, ly, lz, zchunk, nb_wave=296):
    NP = lz + 1
    seen = {}
    for ub, ue in _ranges(lx, ly, lz, zchunk, nb_wave):
        assert ub < ue
        u0 = ub
        while u0 < ue:
            tile = u0 // NP
            zb = u0 - tile * NP
            ze = min(NP, zb + (ue - u0))
            u0 = tile * NP + ze
            H = (ze - zb + L - 1) // L
            for lane in range(L):
                z0 = zb + lane * H - 1
                oend = min(zb + lane * H + H, ze, lz + 1)
                for s in range(H + 2):
                    zs = z0 + s - 1
                    if s >= 2 and zs < oend:
                        key = (tile, zs)
                        seen[key] = seen.get(key, 0) + 1
    return seen


@pytest.mark.parametrize("dims,zchunk,nb", [
    ((256, 128, 128), 22, 296), ((256, 128, 128), -1, 296), ((256, 128, 128), -1, 148),
    ((37, 23, 19), -1, 296), ((37, 23, 19), 5, 296), ((64, 48, 40), -1, 296),
    ((120, 60, 50), -1, 296), ((200, 13, 3), -1, 296), ((5, 3, 1), -1, 296), ((31, 7, 0), -1, 4),
])
def test_every_output_plane_written_once(dims, zchunk, nb):
    lx, ly, lz = dims
    seen = _outputs(lx, ly, lz, zchunk, nb)
    ntx, nty = (lx + TX - 1) // (TX - 1), (ly + TY - 1) // (TY - 1)
    expect = set(itertools.product(range(ntx * nty), range(lz + 1)))
    assert set(seen) == expect
    assert all(v == 1 for v in seen.values())


def test_tma_wait_is_bounded_by_one_second():
    """The TMA pipeline's mbarrier wait (vf_wait.cuh): the suspend-time hint is
    in nanoseconds, and polls x hint stays within the 1 s wall-time limit, so a
    stuck stage cannot hold a CTA longer than about a second."""
    import re
    src = open(os.path.join(REPO, "voxelsim_fea_b200", "csrc", "vf_wait.cuh")).read()

    def const(name):
        m = re.search(name + r"\s*=\s*([0-9]+)u", src)
        assert m, name
        return int(m.group(1))

    hint, polls, limit = const("kPollHintNs"), const("kMaxPolls"), const("kWaitLimitNs")
    assert limit <= 1_000_000_000
    assert hint * polls <= limit
    assert hint <= 10_000          # a poll sleeps at most 10 us


def _trtri_schedule(n, nb=32):
    """The level schedule of the coarsest inverse's batched triangular
    inversion (vf_dense.cu, dense_cholesky_inverse): per level g, the pairs
    (r0, r1, r2) and the scratch offset of each T = L21 Y11."""
    nbk = (n + nb - 1) // nb
    levels = []
    g = 1
    while g < nbk:
        pairs, toff = [], 0
        for p0 in range(0, nbk, 2 * g):
            r0, r1, r2 = p0 * nb, min((p0 + g) * nb, n), min((p0 + 2 * g) * nb, n)
            if r1 >= r2:
                continue
            pairs.append((r0, r1, r2, toff))
            toff += (r2 - r1) * (r1 - r0)
        levels.append((g, pairs, toff))
        g *= 2
    return levels


def test_coarsest_triangular_inversion_schedule():
    """Restated on the host: diagonal 32x32 block inverses, then per level
    Y21 = -Y22 (L21 Y11) over the pairs, give L^-1; the scratch of each level
    fits the n^2 / 2 + 32 n doubles the work buffer reserves."""
    import numpy as np
    rng = np.random.default_rng(0)
    for n in (5, 32, 33, 100, 259, 300):
        L = np.tril(rng.standard_normal((n, n))) + n * np.eye(n)
        Y = np.zeros((n, n))
        for k in range(0, n, 32):
            e = min(k + 32, n)
            Y[k:e, k:e] = np.linalg.inv(L[k:e, k:e])
        for g, pairs, _ in _trtri_schedule(n):
            for r0, r1, r2, _ in pairs:
                T = L[r1:r2, r0:r1] @ Y[r0:r1, r0:r1]
                Y[r1:r2, r0:r1] = -Y[r1:r2, r1:r2] @ T
        np.testing.assert_allclose(Y @ L, np.eye(n), atol=1e-12)
    for n in (5, 33, 4131, 9999, 16384):
        for g, pairs, toff in _trtri_schedule(n):
            assert toff <= n * n // 2 + 32 * n, (n, g, toff)


def _stencil_matrix(nx1, ny1, nz1, R, rng):
    """SPD matrix with the coupling pattern of a reach-R 3x3-block stencil in
    the reference node order r = x + nx1 (y + ny1 z), DOF 3 r + c (the dense
    coarsest operator of vf_dense.cu / vf_wide.cu)."""
    import numpy as np
    n = 3 * nx1 * ny1 * nz1
    A = np.zeros((n, n))
    coords = [(x, y, z) for z in range(nz1) for y in range(ny1) for x in range(nx1)]
    for r, (x, y, z) in enumerate(coords):
        for dz in range(-R, R + 1):
            for dy in range(-R, R + 1):
                for dx in range(-R, R + 1):
                    X, Y, Z = x + dx, y + dy, z + dz
                    if 0 <= X < nx1 and 0 <= Y < ny1 and 0 <= Z < nz1:
                        q = X + nx1 * (Y + ny1 * Z)
                        if q >= r:
                            B = rng.standard_normal((3, 3))
                            A[3 * r:3 * r + 3, 3 * q:3 * q + 3] = B
                            A[3 * q:3 * q + 3, 3 * r:3 * r + 3] = B.T
    # diagonal dominance makes it SPD without changing the pattern
    A += np.diag(np.abs(A).sum(axis=1) + 1.0)
    return A


def test_coarsest_band_limits():
    """The band the coarsest factorization relies on (vf_solver.cu,
    build_dense_coarsest; vf_dense.cu, dense_cholesky_inverse): with
    bw = 3 R (1 + nx1 + nx1 ny1) + 2, a reach-R stencil operator has no entry
    beyond bw; its Cholesky factor has none either (so the panel solve and the
    trailing update of a block column touch only the rows within the band);
    and each L21 block of the triangular inversion's levels, and its product
    T = L21 Y11, is zero below row bw (the rows the batched products skip)."""
    import numpy as np
    rng = np.random.default_rng(1)
    for (nx1, ny1, nz1, R) in [(5, 4, 6, 1), (4, 3, 7, 2), (6, 2, 5, 2)]:
        A = _stencil_matrix(nx1, ny1, nz1, R, rng)
        n = A.shape[0]
        bw = min(3 * R * (1 + nx1 + nx1 * ny1) + 2, n)
        i, j = np.indices(A.shape)
        assert not A[np.abs(i - j) > bw].any()
        Lf = np.linalg.cholesky(A)
        assert not Lf[(i - j) > bw].any()
        Y = np.linalg.inv(Lf)
        for g, pairs, _ in _trtri_schedule(n, nb=8):
            for r0, r1, r2, _ in pairs:
                L21 = Lf[r1:r2, r0:r1]
                assert not L21[bw:].any(), (nx1, ny1, nz1, R, g)
                # the skipped K range of each row tile: L21[a][b] == 0 for b < a + h - bw
                h = r1 - r0
                a, b = np.indices(L21.shape)
                assert not L21[b < a + h - bw].any()
                T = L21 @ Y[r0:r1, r0:r1]
                assert not T[bw:].any()
