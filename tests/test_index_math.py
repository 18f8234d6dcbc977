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


def _ceil_half(v):
    return (v + 1) // 2 if v >= 0 else -((-v) // 2)


def _tw(d):
    return 1.0 if d == 0 else (0.5 if d in (1, -1) else 0.0)


def test_fixed_reach_setup_tables():
    """The compile-time set-up products (vf_wide.cu, k_prolong_blocks_t and
    k_rap_b_t) find the contributing neighbour offsets from per-axis tables;
    restated on the host, they give the same (offset, slot, weight) terms in
    the same order as the generic kernels' scan over all (2R+1)^3 offsets,
    for both reach pairs the hierarchy builds ((R_l, Pr) = (1, 2), (2, 1)),
    at every node of small fine grids (edges and interior)."""
    import itertools
    for RF, PR in [(1, 2), (2, 1)]:
        W, NA, NBA = 2 * RF + 1, PR + 1, PR + RF + 1
        for (lx, ly, lz) in [(6, 4, 4), (5, 3, 7)]:
            cx, cy, cz = lx // 2, ly // 2, lz // 2   # coarse voxels (the grid test uses even and odd)

            def inside_f(x, y, z):
                return 0 <= x <= lx and 0 <= y <= ly and 0 <= z <= lz

            def inside_c(x, y, z):
                return 0 <= x <= cx and 0 <= y <= cy and 0 <= z <= cz

            for x, y, z in itertools.product(range(lx + 1), range(ly + 1), range(lz + 1)):
                # B = A P_s: generic scan (k_rap_b) against the per-axis tables (k_rap_b_t)
                for b in range(NBA ** 3):
                    J = (_ceil_half(x - PR - RF) + b % NBA, _ceil_half(y - PR - RF) + (b // NBA) % NBA,
                         _ceil_half(z - PR - RF) + b // (NBA * NBA))
                    if not inside_c(*J):
                        continue
                    generic = []
                    for s in range(W ** 3):
                        ix, iy, iz = x + s % W - RF, y + (s // W) % W - RF, z + s // (W * W) - RF
                        if not inside_f(ix, iy, iz):
                            continue
                        a = (J[0] - _ceil_half(ix - PR), J[1] - _ceil_half(iy - PR), J[2] - _ceil_half(iz - PR))
                        if min(a) < 0 or max(a) > PR:
                            continue
                        generic.append((s, (a[2] * NA + a[1]) * NA + a[0]))
                    tab = []
                    for axis, (v, hi) in enumerate([(x, lx), (y, ly), (z, lz)]):
                        col = []
                        for d in range(W):
                            iv = v + d - RF
                            av = J[axis] - _ceil_half(iv - PR)
                            col.append(av if (0 <= iv <= hi and 0 <= av <= PR) else -1)
                        tab.append(col)
                    fixed = [(((dz * W) + dy) * W + dx, (tab[2][dz] * NA + tab[1][dy]) * NA + tab[0][dx])
                             for dz in range(W) if tab[2][dz] >= 0
                             for dy in range(W) if tab[1][dy] >= 0
                             for dx in range(W) if tab[0][dx] >= 0]
                    assert fixed == generic, (RF, PR, x, y, z, b)
                # P_s blocks: generic weights (k_prolong_blocks) against per-axis weights
                for slot in range(NA ** 3):
                    J = (_ceil_half(x - PR) + slot % NA, _ceil_half(y - PR) + (slot // NA) % NA,
                         _ceil_half(z - PR) + slot // (NA * NA))
                    if not inside_c(*J):
                        continue
                    generic = []
                    for s in range(W ** 3):
                        dx, dy, dz = s % W - RF, (s // W) % W - RF, s // (W * W) - RF
                        wk = _tw(x + dx - 2 * J[0]) * _tw(y + dy - 2 * J[1]) * _tw(z + dz - 2 * J[2])
                        if wk == 0.0 or not inside_f(x + dx, y + dy, z + dz):
                            continue
                        generic.append((s, wk))
                    wts = []
                    for axis, (v, hi) in enumerate([(x, lx), (y, ly), (z, lz)]):
                        wts.append([(_tw(v + d - RF - 2 * J[axis]) if 0 <= v + d - RF <= hi else 0.0)
                                    for d in range(W)])
                    fixed = [(((dz * W) + dy) * W + dx, wts[0][dx] * wts[1][dy] * wts[2][dz])
                             for dz in range(W) if wts[2][dz] != 0.0
                             for dy in range(W) if wts[1][dy] != 0.0
                             for dx in range(W) if wts[0][dx] != 0.0]
                    assert fixed == generic, (RF, PR, x, y, z, slot)
