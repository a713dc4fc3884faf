"""The drop-in boundary on CPU: record layouts, the C-ABI library's exports,
the host planner and host-side validation.  No CUDA device needed."""

import ctypes
import os
import re

import numpy as np
import pytest

from forcepho_b200 import _native as N
from forcepho_b200 import kernel_limits as K
from forcepho_b200 import structs
from forcepho_b200 import synthetic as S

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "forcepho_b200.h")


def test_limits_match_reference_values():
    # forcepho/src/kernel_limits.h:5-26
    assert (K.MAXBANDS, K.MAXSOURCES, K.NPARAMS, K.MAX_EXP_ARG, K.MAXRADII) == (30, 30, 7, 36.0, 10)


def test_struct_sizes():
    assert structs.patch_struct_dtype.itemsize == 152
    assert structs.source_struct_dtype.itemsize == 264
    assert structs.response_struct_dtype.itemsize == 840
    assert structs.psf_dtype.itemsize == 28
    # field offsets of the patch struct (forcepho/src/patch.cc:23-100)
    off = {n: structs.patch_struct_dtype.fields[n][1] for n in structs.patch_struct_dtype.names}
    assert off["n_sources"] == 72 and off["n_radii"] == 76 and off["rad2"] == 80 and off["psfgauss_start"] == 144


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"FP_API[^;(]*?\b(fp_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = N.load()
    syms = declared_symbols()
    assert len(syms) >= 9
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(N.SIGNATURES), "binding signatures and header disagree"


def test_normal_library_has_no_phase_timers():
    """The clock64 phase counters exist only in the diagnostic build
    (``python -m forcepho_b200.build --phase-timers``)."""
    L = N.load()
    assert not hasattr(L, "fp_debug_phases")


def test_struct_sizes_reported_by_library():
    L = N.load()
    out = np.zeros(4, np.int32)
    assert L.fp_struct_sizes(out.ctypes.data) == 0
    assert list(out) == [152, 264, 840, 28]


def plan(patches, tile, coordinates=True):
    L = N.load()
    shapes = [N.patch_shape(p, coordinates=coordinates) for p in patches]
    arr = (N.PatchShape * len(shapes))(*shapes)
    sz = N.PlanSizes()
    rc = L.fp_plan_count(ctypes.addressof(arr), len(shapes), tile, ctypes.byref(sz))
    if rc:
        return rc, None
    ex = np.zeros(sz.n_exposures, N.exposure_desc_dtype)
    ti = np.zeros(sz.n_tiles, N.tile_dtype)
    bd = np.zeros(sz.n_band_outputs, N.band_desc_dtype)
    od = np.zeros(sz.n_tiles, np.int32)
    pm = np.zeros(sz.n_perm, np.int32)
    N.check(L.fp_plan_fill(ctypes.addressof(arr), len(shapes), tile, ex.ctypes.data, ti.ctypes.data,
                           bd.ctypes.data, od.ctypes.data, pm.ctypes.data), "fill")
    return 0, (sz, ex, ti, bd, od, pm)


CELL = {1024: (32, 32), 512: (32, 16), 256: (16, 16)}


@pytest.mark.parametrize("tile", [256, 512, 1024])
@pytest.mark.parametrize("coordinates", [True, False])
def test_planner_tables(tile, coordinates):
    patches = S.config_batched(seed=7, n_patches=6)
    rc, (sz, ex, ti, bd, od, pm) = plan(patches, tile, coordinates)
    assert rc == 0
    assert sz.n_pairs == sum(p.n_pairs() for p in patches)
    assert sz.n_exposures == sum(p.n_exp for p in patches)
    assert sz.n_band_outputs == sum(p.n_bands for p in patches)
    assert sz.n_perm == sum(p.npix for p in patches)
    k = 0
    for pi, p in enumerate(patches):
        ns = int(p.n_sources)
        for b in range(p.n_bands):
            e0, ne = int(p.band_start[b]), int(p.band_N[b])
            row = bd[[i for i in range(len(bd)) if bd["patch"][i] == pi and bd["band"][i] == b][0]]
            assert row["tile_begin"] == k and row["n_sources"] == ns
            for e in range(e0, e0 + ne):
                s0, n = int(p.exposure_start[e]), int(p.exposure_N[e])
                seen = []
                while len(seen) < n:
                    t = ti[k]
                    assert ex[t["expo"]]["patch"] == pi and ex[t["expo"]]["exposure"] == e
                    assert 0 < t["n_pix"] <= tile
                    pix = pm[t["perm_start"]:t["perm_start"] + t["n_pix"]]
                    assert np.all((pix >= s0) & (pix < s0 + n))
                    if coordinates:
                        x, y = p.xpix[pix], p.ypix[pix]
                        if np.all(x >= 0):      # a real cell (the pad pixels share their own)
                            cw, ch = CELL[tile]
                            assert x.max() - x.min() < cw and y.max() - y.min() < ch
                    else:
                        assert np.array_equal(pix, np.arange(s0 + len(seen), s0 + len(seen) + len(pix)))
                    seen.extend(pix.tolist())
                    k += 1
                # every pixel of the exposure exactly once
                assert sorted(seen) == list(range(s0, s0 + n))
            assert row["tile_end"] == k
    assert k == sz.n_tiles
    stride = np.array([1 + 7 * ex[t["expo"]]["n_sources"] for t in ti])
    assert np.array_equal(ti["partial_offset"], np.concatenate([[0], np.cumsum(stride)[:-1]]))
    assert sz.n_partials == stride.sum()
    assert sorted(od.tolist()) == list(range(sz.n_tiles))
    work = ti["n_pix"][od].astype(np.int64) * ex[ti["expo"][od]]["n_gauss"]
    assert np.all(np.diff(work) <= 0)


def test_planner_sparse_and_nonfinite_coordinates():
    """Far-apart pixels (sparse grid, sorted path) and non-finite coordinates
    still yield every pixel exactly once."""
    p = S.config_small(seed=1)
    p.xpix = p.xpix.copy()
    p.ypix = p.ypix.copy()
    p.xpix[::97] *= 1e6
    p.xpix[5] = np.nan
    p.ypix[7] = np.inf
    rc, (sz, ex, ti, bd, od, pm) = plan([p], 256)
    assert rc == 0
    assert sorted(pm.tolist()) == list(range(p.npix))
    assert ti["n_pix"].sum() == p.npix


def test_planner_extreme_finite_coordinates():
    """Coordinates near the float range (cell counts far past int64 if not
    clamped) still yield every pixel exactly once."""
    p = S.config_small(seed=1)
    p.xpix = p.xpix.copy()
    p.ypix = p.ypix.copy()
    p.xpix[3] = 3.0e38
    p.ypix[11] = -3.0e38
    p.xpix[20] = -1.0e30
    rc, (sz, ex, ti, bd, od, pm) = plan([p], 256)
    assert rc == 0
    assert sorted(pm.tolist()) == list(range(p.npix))
    assert ti["n_pix"].sum() == p.npix


def test_planner_rejects_bad_shapes():
    p = S.config_small(seed=1)
    assert plan([p], 100)[0] == N.FP_ERR_ARGUMENT          # not a multiple of 32
    bad = S.config_small(seed=1)
    bad.exposure_N = bad.exposure_N + 64          # past the end of the pixel arrays
    assert plan([bad], 256)[0] == N.FP_ERR_ARGUMENT
    assert "outside" in N.load().fp_error_string().decode()


def test_validate_rejects_inconsistent_patch():
    p = S.config_multiband(seed=2, n_sources=3, n_bands=2, exp_per_band=2, size=40)
    assert p.validate()
    q = S.config_multiband(seed=2, n_sources=3, n_bands=2, exp_per_band=2, size=40)
    q.band_N = q.band_N.copy()
    q.band_N[0] = 3
    with pytest.raises(ValueError):
        q.validate()
    r = S.config_multiband(seed=2, n_sources=3, n_bands=2, exp_per_band=2, size=40)
    r.psfgauss = r.psfgauss.copy()
    r.psfgauss["sersic_bin"][0] = 12
    with pytest.raises(ValueError):
        r.validate()


def test_planner_tile_rule_classes():
    """A tile rule gives each exposure the tile size of its pixel-count class;
    each tile records its class, and every pixel appears exactly once."""
    L = N.load()
    patches = S.config_batched(seed=9, n_patches=8)
    shapes = [N.patch_shape(p) for p in patches]
    arr = (N.PatchShape * len(shapes))(*shapes)
    classes = [(4096, 256), (16384, 512), (1 << 30, 1024)]
    rule = N.tile_rule(classes)
    sz = N.PlanSizes()
    N.check(L.fp_plan_count_rule(ctypes.addressof(arr), len(shapes), ctypes.byref(rule), ctypes.byref(sz)), "count")
    ex = np.zeros(sz.n_exposures, N.exposure_desc_dtype)
    ti = np.zeros(sz.n_tiles, N.tile_dtype)
    bd = np.zeros(sz.n_band_outputs, N.band_desc_dtype)
    od = np.zeros(sz.n_tiles, np.int32)
    pm = np.zeros(sz.n_perm, np.int32)
    N.check(L.fp_plan_fill_rule(ctypes.addressof(arr), len(shapes), ctypes.byref(rule), ex.ctypes.data,
                                ti.ctypes.data, bd.ctypes.data, od.ctypes.data, pm.ctypes.data), "fill")
    seen_classes = set()
    for t in ti:
        e = ex[t["expo"]]
        p = patches[e["patch"]]
        n = int(p.exposure_N[e["exposure"]])
        want = 256 if n <= 4096 else (512 if n <= 16384 else 1024)
        assert t["tile_pixels"] == want and 0 < t["n_pix"] <= want
        seen_classes.add(want)
    assert seen_classes == {256, 512, 1024}
    off = 0
    for p in patches:
        assert sorted(pm[off:off + p.npix].tolist()) == list(range(p.npix))
        off += p.npix
    # a single tile size is the one-class rule
    sz1 = N.PlanSizes()
    N.check(L.fp_plan_count(ctypes.addressof(arr), len(shapes), 512, ctypes.byref(sz1)), "count")
    sz2 = N.PlanSizes()
    N.check(L.fp_plan_count_rule(ctypes.addressof(arr), len(shapes), ctypes.byref(N.tile_rule([(0, 512)])),
                                 ctypes.byref(sz2)), "count")
    assert sz1.n_tiles == sz2.n_tiles and sz1.n_partials == sz2.n_partials
    odd = N.tile_rule([(4096, 256), (16384, 768)])       # a multiple of 32 the kernel does not run
    assert L.fp_plan_count_rule(ctypes.addressof(arr), len(shapes), ctypes.byref(odd), ctypes.byref(sz)) \
        == N.FP_ERR_ARGUMENT
    bad = N.tile_rule([(4096, 256), (16384, 500)])
    assert L.fp_plan_count_rule(ctypes.addressof(arr), len(shapes), ctypes.byref(bad), ctypes.byref(sz)) \
        == N.FP_ERR_ARGUMENT


def test_f64_entry_point_rejects_bad_arguments():
    """fp_evaluate_proposal_f64 checks its arguments on the host, before any
    CUDA call: the pointers here are never dereferenced."""
    import ctypes
    from forcepho_b200 import _native as N
    from forcepho_b200.kernel_limits import MAXBANDS
    L = N.load()
    n = ctypes.c_size_t()
    assert L.fp_f64_workspace_bytes(3, 40, ctypes.byref(n)) == N.FP_OK
    assert n.value >= 256 + 3 * 40 and n.value % 256 == 0
    assert L.fp_f64_workspace_bytes(-1, 40, ctypes.byref(n)) == N.FP_ERR_ARGUMENT
    fake, ws = ctypes.c_void_p(4096), ctypes.c_void_p(8192)

    def call(n_bands=2, n_exp=3, ws_ptr=ws, ws_bytes=n.value):
        return L.fp_evaluate_proposal_f64(fake, fake, n_bands, n_exp, 40, fake, fake, ws_ptr, ws_bytes, None)

    assert L.fp_f64_workspace_bytes(3, 40, ctypes.byref(n)) == N.FP_OK
    assert call(n_bands=0) == N.FP_ERR_LIMITS
    assert call(n_bands=MAXBANDS + 1) == N.FP_ERR_LIMITS
    assert call(ws_ptr=ctypes.c_void_p(8192 + 16)) == N.FP_ERR_ARGUMENT
    assert call(ws_bytes=n.value - 1) == N.FP_ERR_WORKSPACE
    assert b"workspace" in L.fp_error_string()
    assert L.fp_evaluate_proposal_f64(None, fake, 2, 3, 40, fake, fake, ws, n.value, None) == N.FP_ERR_ARGUMENT
