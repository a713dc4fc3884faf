"""CPU replay of the tile kernel's adjoint work partition (forcepho_b200/csrc/tiled.cu).

The (group of 32 Gaussians) x (nonzero pixel) plane of one chunk is split
evenly over the 8 warps; warp w writes its segment of group g into slot group
g + w, and the per-source reduction sums, for group g, the slot groups g + w
of exactly the warps whose share meets row g (a bit mask per group, computed
once per chunk).  This replays that integer arithmetic and checks that every
(group, pixel) unit is summed exactly once, that no two segments share a slot
(so every slot read was written in the same chunk), and that the source ranges
found without integer division are the ones division gives."""

import itertools

import pytest

WARPS = 8
CHUNK = 128
SLOT_GROUPS = CHUNK // 32 + WARPS - 1


def segments(ngrp, nzt):
    W = ngrp * nzt
    segs = []      # (warp, group, p0, p1, slot)
    for w in range(WARPS):
        u, u1 = W * w // WARPS, W * (w + 1) // WARPS
        while u < u1:
            grp = u // nzt
            p0 = u - grp * nzt
            p1 = min(nzt, p0 + (u1 - u))
            segs.append((w, grp, p0, p1, grp + w))
            u += p1 - p0
    return segs


def group_mask(ngrp, nzt, grp):
    W = ngrp * nzt
    r0, r1 = grp * nzt, grp * nzt + nzt
    mask = 0
    for w in range(WARPS):
        a, b = W * w // WARPS, W * (w + 1) // WARPS
        if a < b and a < r1 and b > r0:
            mask |= 1 << w
    return mask


def reader_slots(ngrp, nzt, grp):
    m = group_mask(ngrp, nzt, grp)
    out = []
    while m:                                    # lowest set bit first, as __ffs
        w = (m & -m).bit_length() - 1
        m &= m - 1
        out.append(grp + w)
    return out


@pytest.mark.parametrize("ngrp,nzt", list(itertools.product(range(1, CHUNK // 32 + 1),
                                                            [1, 2, 3, 7, 8, 31, 32, 33, 100, 255, 256,
                                                             257, 511, 1000, 1023, 1024])))
def test_partition_covers_plane_once(ngrp, nzt):
    segs = segments(ngrp, nzt)
    slots = [s[4] for s in segs]
    assert len(slots) == len(set(slots)), "two segments share a slot"
    assert max(slots) < SLOT_GROUPS
    by_slot = {s[4]: s for s in segs}
    for g in range(ngrp):
        covered = []
        for sl in reader_slots(ngrp, nzt, g):
            w, grp, p0, p1, _ = by_slot[sl]
            assert grp == g, "reader takes another group's segment"
            covered.extend(range(p0, p1))
        assert sorted(covered) == list(range(nzt))


def _search(keys, lo, hi, pred):
    while lo < hi:
        mid = (lo + hi) >> 1
        if pred(keys[mid]):
            lo = mid + 1
        else:
            hi = mid
    return lo


@pytest.mark.parametrize("n_psf", [1, 3, 4, 36, 40])
def test_source_ranges_without_division(n_psf):
    import numpy as np
    rng = np.random.default_rng(n_psf)
    for _ in range(50):
        ns = int(rng.integers(1, 31))
        kept = np.sort(rng.choice(ns * n_psf, size=int(rng.integers(1, min(CHUNK, ns * n_psf) + 1)),
                                  replace=False))
        for s in range(ns):
            lo_div = _search(kept, 0, len(kept), lambda g: g // n_psf < s)
            end_div = _search(kept, lo_div, len(kept), lambda g: g // n_psf <= s)
            lo = _search(kept, 0, len(kept), lambda g: g < s * n_psf)
            end = _search(kept, lo, len(kept), lambda g: g < (s + 1) * n_psf)
            assert (lo, end) == (lo_div, end_div)
            assert all(g // n_psf == s for g in kept[lo:end])
