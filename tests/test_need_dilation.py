"""The incremental update's dilation of dirty blocks, restated on the CPU.

need_body (egg-sync_b200/csrc/egg_update.cu) widens every dirty block b of
dimension od (zblk cells each, nzb blocks, nzb <= 64) to the blocks holding
the cells [b*zblk - r - 1, (b+1)*zblk - 1 + r + 1], clipped to the grid, in
closed form: bits b - ceil((r+1)/zblk) .. b + 1 + floor(r/zblk) of the mask.
This checks the closed form against the per-block interval union on the
geometries the reference's formulas give (the oracle's geometry) and on
every small width."""
import numpy as np
import pytest

from oracle import Oracle


def blocks(width, od, d):
    """zblk, nzb as the library lays them out."""
    if od < d:
        zblk = max(1, (width + 63) // 64)
        return zblk, (width + zblk - 1) // zblk
    return width, 1


def by_interval(m, zblk, r, width):
    out = 0
    for b in range(64):
        if (m >> b) & 1:
            lo = max(0, b * zblk - r - 1)
            hi = min(width - 1, (b + 1) * zblk - 1 + r + 1)
            for k in range(lo // zblk, hi // zblk + 1):
                out |= 1 << k
    return out


def closed_form(m, zblk, nzb, r):
    lo_sh = min(63, (r + zblk) // zblk)
    hi_sh = min(63, 1 + r // zblk)
    full = (1 << 64) - 1 if nzb >= 64 else (1 << nzb) - 1
    out = 0
    for s in range(lo_sh + 1):
        out |= m >> s
    for s in range(1, hi_sh + 1):
        out |= (m << s) & ((1 << 64) - 1)
    return out & full


def masks(nzb, rng, count=40):
    yield 1
    yield 1 << (nzb - 1)
    yield (1 << nzb) - 1
    for _ in range(count):
        yield int(rng.integers(0, 1 << min(nzb, 62))) | (int(rng.integers(0, 2)) << (nzb - 1))


@pytest.mark.parametrize("n,d,eps", [(1_000_000, 3, 0.015), (500_000, 3, 0.02), (20_000, 16, 0.15), (10_000, 2, 0.05),
                                     (250_000, 3, 0.03), (100_000, 5, 0.08), (1_000, 2, 0.01), (200_000, 1, 0.001),
                                     (4_839, 5, 0.05), (45_781, 3, 0.05)])
def test_closed_form_on_reference_geometries(n, d, eps):
    g = Oracle().geometry(n, d, eps)
    zblk, nzb = blocks(g.width, g.od, d)
    rng = np.random.default_rng(n + d)
    for m in masks(nzb, rng):
        assert closed_form(m, zblk, nzb, g.r) == by_interval(m, zblk, g.r, g.width)


def test_closed_form_on_small_widths():
    rng = np.random.default_rng(7)
    for width in range(2, 300):
        for od, d in ((1, 2), (2, 2)):
            zblk, nzb = blocks(width, od, d)
            for r in range(0, 10):
                for m in masks(nzb, rng, 6):
                    assert closed_form(m, zblk, nzb, r) == by_interval(m, zblk, r, width)


def zwindow_mask(width, zblk, zl, zh):
    """egg_stencil.cuh zwindow_mask: bits of the blocks meeting cells [zl, zh]."""
    bl, bh = max(0, zl) // zblk, min(width - 1, zh) // zblk
    return ((2 << bh) - (1 << bl)) & ((1 << 64) - 1)


@pytest.mark.parametrize("n,d,eps", [(1_000_000, 3, 0.015), (20_000, 16, 0.15), (100_000, 5, 0.08), (45_781, 3, 0.05)])
def test_column_mask_never_hides_a_candidate(n, d, eps):
    """A column is passed over only when no cell of it lies in the lane's
    window [z - r - 1, z + r + 1] (the range its two binary searches cover)."""
    g = Oracle().geometry(n, d, eps)
    if g.od >= d:
        pytest.skip("no inner dimension")
    zblk, nzb = blocks(g.width, g.od, d)
    rng = np.random.default_rng(n)
    for _ in range(300):
        cells = np.unique(rng.integers(0, g.width, int(rng.integers(0, 12))))
        colmask = 0
        for z in cells:
            colmask |= 1 << int(z // zblk)
        z = int(rng.integers(0, g.width))
        zl, zh = z - g.r - 1, z + g.r + 1
        has = bool(((cells >= zl) & (cells <= zh)).any())
        passes = (colmask & zwindow_mask(g.width, zblk, zl, zh)) != 0
        assert passes or not has
