"""CPU replay of the tile kernel's adjoint work partition (forcepho_b200/csrc/tiled.cu).

The (group of 32 Gaussians) x (nonzero pixel) plane of one chunk is split
evenly over the 8 warps; a warp walks its share as segments, one per group
row it meets.  After each segment the warp sums its lanes' gradients per
source with a segmented shuffle tree (a source's Gaussians occupy contiguous
lanes, invalid lanes carry source -1) and the first lane of each source adds
the sum into the warp's own row of per-source gradients; the rows of the 8
warps are summed once per tile.  This replays that integer arithmetic and
checks that every (group, pixel) unit is processed exactly once and that the
shuffle tree leaves each source's exact sum on its first lane."""

import itertools

import numpy as np
import pytest

WARPS = 8
CHUNK = 256


def segments(ngrp, nzt):
    W = ngrp * nzt
    segs = []      # (warp, group, p0, p1)
    for w in range(WARPS):
        u, u1 = W * w // WARPS, W * (w + 1) // WARPS
        while u < u1:
            grp = u // nzt
            p0 = u - grp * nzt
            p1 = min(nzt, p0 + (u1 - u))
            segs.append((w, grp, p0, p1))
            u += p1 - p0
    return segs


@pytest.mark.parametrize("ngrp,nzt", list(itertools.product(range(1, CHUNK // 32 + 1),
                                                            [1, 2, 3, 7, 8, 31, 32, 33, 100, 255, 256,
                                                             257, 511, 1000, 1023, 1024])))
def test_partition_covers_plane_once(ngrp, nzt):
    covered = {g: [] for g in range(ngrp)}
    for w, grp, p0, p1 in segments(ngrp, nzt):
        assert 0 <= p0 < p1 <= nzt
        covered[grp].extend(range(p0, p1))
    for g in range(ngrp):
        assert sorted(covered[g]) == list(range(nzt))


def segmented_lane_sums(src, val):
    """The kernel's shuffle tree: lane l adds lane l+o's value (read before this
    step) when l+o < 32 and both lanes hold the same source."""
    v = list(val)
    for o in (1, 2, 4, 8, 16):
        prev = list(v)
        for lane in range(32):
            if lane + o < 32 and src[lane + o] == src[lane]:
                v[lane] = prev[lane] + prev[lane + o]
    heads = {}
    for lane in range(32):
        if src[lane] >= 0 and (lane == 0 or src[lane - 1] != src[lane]):
            heads[src[lane]] = v[lane]
    return heads


@pytest.mark.parametrize("seed", range(40))
def test_segmented_shuffle_sums(seed):
    rng = np.random.default_rng(seed)
    n_valid = int(rng.integers(1, 33))
    # ascending sources over the valid lanes, -1 on the rest
    src = sorted(int(s) for s in rng.integers(0, int(rng.integers(1, 31)), n_valid)) + [-1] * (32 - n_valid)
    val = [int(x) for x in rng.integers(-1000, 1000, 32)]
    heads = segmented_lane_sums(src, val)
    want = {}
    for s, x in zip(src, val):
        if s >= 0:
            want[s] = want.get(s, 0) + x
    assert heads == want


@pytest.mark.parametrize("ngrp,nzt,n_psf", [(1, 5, 4), (2, 300, 36), (4, 1024, 36), (3, 33, 7), (4, 1, 36)])
def test_every_unit_reaches_its_source_once(ngrp, nzt, n_psf):
    """Integer stand-ins for the per-(Gaussian, pixel) gradient terms: the per-warp
    source rows, summed over warps, equal the direct per-source sums."""
    rng = np.random.default_rng(ngrp * 1000 + nzt)
    cn = min(CHUNK, ngrp * 32 - int(rng.integers(0, 32)))
    cn = max(cn, (ngrp - 1) * 32 + 1)
    gidx = np.sort(rng.choice(30 * n_psf, size=cn, replace=False))
    term = rng.integers(-50, 50, size=(cn, nzt))
    rows = np.zeros((WARPS, 30), dtype=np.int64)
    for w, grp, p0, p1 in segments(ngrp, nzt):
        src = [int(gidx[grp * 32 + l]) // n_psf if grp * 32 + l < cn else -1 for l in range(32)]
        val = [int(term[grp * 32 + l, p0:p1].sum()) if grp * 32 + l < cn else 0 for l in range(32)]
        for s, x in segmented_lane_sums(src, val).items():
            rows[w, s] += x
    want = np.zeros(30, dtype=np.int64)
    for i in range(cn):
        want[gidx[i] // n_psf] += term[i].sum()
    np.testing.assert_array_equal(rows.sum(axis=0), want)
