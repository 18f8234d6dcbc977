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


def _ceil_half(v):
    return -((-v) // 2)


def _offset_range(lo, hi, R, x, lmax):
    return max(lo, -R, -x), min(hi, R, lmax - x)


def test_wide_setup_offset_ranges():
    """The smoothed-transfer set-up kernels (vf_wide.cu) loop only over the
    neighbour offsets that can contribute; restated here against a scan of all
    offsets with the kernels' own skip tests, per axis, over every fine
    position, coarse slot and reach in use: the same offsets, in order."""
    import itertools as it
    for (Pr, Rf) in ((2, 1), (1, 2), (1, 1)):
        for lmax in (6, 9):
            lc = lmax // 2
            for x in range(lmax + 1):
                for J in range(lc + 1):
                    # k_rap_b: i = x + d with ceil((i - Pr) / 2) in [J - Pr, J], d in [-Rf, Rf], i inside
                    full = [d for d in range(-Rf, Rf + 1) if 0 <= x + d <= lmax
                            and 0 <= J - _ceil_half(x + d - Pr) <= Pr]
                    a, b = _offset_range(2 * J - Pr - 1 - x, 2 * J + Pr - x, Rf, x, lmax)
                    assert full == list(range(a, b + 1)), (Pr, Rf, x, J)
                    # k_prolong_blocks: |x + d - 2J| <= 1
                    full = [d for d in range(-Rf, Rf + 1) if 0 <= x + d <= lmax and abs(x + d - 2 * J) <= 1]
                    a, b = _offset_range(2 * J - x - 1, 2 * J - x + 1, Rf, x, lmax)
                    assert full == list(range(a, b + 1)), (Pr, Rf, x, J)
            for X, J in it.product(range(lc + 1), range(lc + 1)):
                # k_rap_c: i = 2X + o, |o| <= Pr, ceil((i - Pr - Rf) / 2) in [J - Pr - Rf, J], i inside
                full = [o for o in range(-Pr, Pr + 1) if 0 <= 2 * X + o <= lmax
                        and 0 <= J - _ceil_half(2 * X + o - Pr - Rf) <= Pr + Rf]
                a, b = _offset_range(2 * J - Pr - Rf - 1 - 2 * X, 2 * J + Pr + Rf - 2 * X, Pr, 2 * X, lmax)
                assert full == list(range(a, b + 1)), (Pr, Rf, X, J)
