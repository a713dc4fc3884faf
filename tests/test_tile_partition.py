"""CPU replay of the tile kernel's adjoint work partition (forcepho_b200/csrc/tiled.cu).

The (group of 32 Gaussians) x (nonzero pixel) plane of one chunk is split
evenly over the 8 warps; a warp walks its share as segments, one per group
row it meets.  A chunk's last group of v < 32 Gaussians is replicated
k = min(8, 32 // v) times over the lanes (lane = replica * v + Gaussian), each
replica taking every k-th pixel, so that group has ceil(nzt / k) units of k
pixels; a fixed shuffle tree sums the replicas into replica 0.  After each
segment the warp sums its lanes' gradients per source with a segmented shuffle
tree (a source's Gaussians occupy contiguous lanes, other lanes carry source
-1) and the first lane of each source adds the sum into the warp's own row of
per-source gradients; the rows of the 8 warps are summed once per tile.  This
replays that integer arithmetic and checks that every (Gaussian, pixel) pair
reaches its Gaussian's replica-0 lane exactly once, that every pixel index
stays inside the tile, and that the shuffle tree leaves each source's exact
sum on its first lane."""

import numpy as np
import pytest

WARPS = 8
CHUNK = 256          # Gaussians per chunk: at most 8 groups
MAX_REPLICAS = 8


def layout(cn, nzt):
    """The chunk's partition constants: groups, Gaussians in the last group,
    its replicas, its units, units of the full groups."""
    ngrp = (cn + 31) >> 5
    vlast = cn - ((ngrp - 1) << 5)
    krep = min(MAX_REPLICAS, 32 // vlast)
    ulast = (nzt + krep - 1) // krep
    return ngrp, vlast, krep, ulast, (ngrp - 1) * nzt


def segments(cn, nzt):
    """(warp, group, q0, q1) of every segment, in units of the group's row."""
    ngrp, vlast, krep, ulast, ufull = layout(cn, nzt)
    W = ufull + ulast
    segs = []
    for w in range(WARPS):
        u, u1 = W * w // WARPS, W * (w + 1) // WARPS
        while u < u1:
            if u < ufull:
                grp, q0, qn = u // nzt, u - (u // nzt) * nzt, nzt
            else:
                grp, q0, qn = ngrp - 1, u - ufull, ulast
            q1 = min(qn, q0 + (u1 - u))
            segs.append((w, grp, q0, q1))
            u += q1 - q0
    return segs


def lane_pixels(cn, nzt, grp, q0, q1):
    """Per lane: (Gaussian index or None, replica, pixel indices it walks)."""
    ngrp, vlast, krep, _, _ = layout(cn, nzt)
    kr, vg = (krep, vlast) if grp == ngrp - 1 else (1, 32)
    out = []
    for lane in range(32):
        rep = lane // vg
        gl = grp * 32 + lane - rep * vg
        valid = rep < kr and gl < cn
        if kr == 1:
            ps = range(q0, q1)
        else:
            pe = min(nzt, q1 * kr)
            ps = range(q0 * kr + rep if valid else pe, pe, kr)
        out.append((gl if valid else None, rep, list(ps)))
    return out, kr, vg


def replica_tree(vals, kr, vg):
    """The kernel's replica sum: at step o, lane (rep, i) adds lane (rep + o, i)
    (read before this step) when rep is a multiple of 2o and rep + o < kr."""
    v = list(vals)
    o = 1
    while o < kr:
        prev = list(v)
        for lane in range(32):
            rep = lane // vg
            if (rep & (2 * o - 1)) == 0 and rep + o < kr:
                v[lane] = prev[lane] + prev[lane + o * vg]
        o <<= 1
    return v


@pytest.mark.parametrize("cn", list(range(1, 33)) + [33, 40, 63, 64, 65, 100, 127, 200, 224, 225, 255, CHUNK])
@pytest.mark.parametrize("nzt", [1, 2, 3, 7, 8, 9, 31, 32, 33, 100, 255, 256, 257, 511, 1000, 1023, 1024])
def test_partition_covers_plane_once(cn, nzt):
    count = np.zeros((cn, nzt), dtype=np.int64)
    for w, grp, q0, q1 in segments(cn, nzt):
        assert q0 < q1
        lanes, kr, vg = lane_pixels(cn, nzt, grp, q0, q1)
        pairs = [[] for _ in range(32)]
        for lane, (g, rep, ps) in enumerate(lanes):
            assert all(0 <= p < nzt for p in ps)
            if g is not None:
                pairs[lane] = [(g, p) for p in ps]
        tot = replica_tree(pairs, kr, vg)
        for lane, (g, rep, _) in enumerate(lanes):
            if g is not None and rep == 0:
                for gg, p in tot[lane]:
                    assert gg == g
                    count[gg, p] += 1
    assert (count == 1).all()


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


@pytest.mark.parametrize("cn,nzt,n_psf", [(5, 5, 4), (40, 300, 36), (128, 1024, 36), (70, 33, 7),
                                           (100, 1, 36), (3, 1000, 36), (9, 257, 9), (256, 1024, 36)])
def test_every_unit_reaches_its_source_once(cn, nzt, n_psf):
    """Integer stand-ins for the per-(Gaussian, pixel) gradient terms: the per-warp
    source rows, summed over warps, equal the direct per-source sums."""
    rng = np.random.default_rng(cn * 1000 + nzt)
    gidx = np.sort(rng.choice(30 * n_psf, size=cn, replace=False))
    term = rng.integers(-50, 50, size=(cn, nzt))
    rows = np.zeros((WARPS, 30), dtype=np.int64)
    for w, grp, q0, q1 in segments(cn, nzt):
        lanes, kr, vg = lane_pixels(cn, nzt, grp, q0, q1)
        val = [int(term[g, ps].sum()) if g is not None else 0 for g, _, ps in lanes]
        val = replica_tree(val, kr, vg)
        src = [int(gidx[g]) // n_psf if g is not None and rep == 0 else -1 for g, rep, _ in lanes]
        val = [x if s >= 0 else 0 for x, s in zip(val, src)]
        for s, x in segmented_lane_sums(src, val).items():
            rows[w, s] += x
    want = np.zeros(30, dtype=np.int64)
    for i in range(cn):
        want[gidx[i] // n_psf] += term[i].sum()
    np.testing.assert_array_equal(rows.sum(axis=0), want)
