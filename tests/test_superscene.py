"""The scene bookkeeping (forcepho_b200.superscene) against golden checkouts made
by the reference's own SuperScene / LinkedSuperScene code
(tests/golden/make_superscene_golden.py), plus the properties of the sky-offset
frame and the catalog/bounds helpers."""

import json
import os

import numpy as np
import pytest

from forcepho_b200 import superscene as SS
from forcepho_b200.stores import fits as F

GOLD = os.path.join(os.path.dirname(__file__), "golden", "superscene_golden.json")
SEEDS = [0, 7, 19, 33, 7, 58, 101, 150, 151, 222, 305, 399, 12, 64]


@pytest.fixture(scope="module")
def gold():
    with open(GOLD) as f:
        return json.load(f)


def catalog(gold):
    bands = gold["bands"]
    c = gold["catalog"]
    cat = np.zeros(len(c["ra"]), dtype=SS.sourcecat_dtype(bands=bands))
    for k in cat.dtype.names:
        cat[k] = c[k]
    return cat, bands


def test_offset_frame_matches_the_rotation_of_the_fixture(gold):
    cat, bands = catalog(gold)
    sc = SS.SuperScene(sourcecat=cat, bands=bands)
    np.testing.assert_allclose(sc.scene_coordinates, np.array(gold["circular"]["scene_coordinates"]),
                               rtol=0, atol=1e-8)


def test_offset_frame_properties():
    ra0, dec0 = 150.2, 2.3
    x, y = SS.sky_to_offset(ra0, dec0, ra0, dec0)
    assert abs(x) < 1e-9 and abs(y) < 1e-9
    # along the meridian through the origin: lon 0, lat the declination offset
    x, y = SS.sky_to_offset(ra0, dec0 + 0.01, ra0, dec0)
    assert abs(x) < 1e-9 and abs(y - 36.0) < 1e-8
    # small offsets: lon = dRA cos(dec0)
    x, y = SS.sky_to_offset(ra0 + 1e-4, dec0, ra0, dec0)
    assert abs(x - 0.36 * np.cos(np.deg2rad(dec0))) < 1e-6 and abs(y) < 1e-6
    # the separation from the origin is preserved
    rng = np.random.default_rng(3)
    ra, dec = ra0 + rng.uniform(-2, 2, 50), dec0 + rng.uniform(-2, 2, 50)
    x, y = SS.sky_to_offset(ra, dec, ra0, dec0)
    lon, lat = np.deg2rad(x / 3600), np.deg2rad(y / 3600)
    a, d, a0, d0 = map(np.deg2rad, (ra, dec, ra0, dec0))
    sep = np.arccos(np.sin(d) * np.sin(d0) + np.cos(d) * np.cos(d0) * np.cos(a - a0))
    np.testing.assert_allclose(np.arccos(np.cos(lat) * np.cos(lon)), sep, atol=1e-12)


def _run_checkouts(sc, bands, circular):
    out, held = [], []
    for k, s in enumerate(SEEDS):
        region, active, fixed = sc.checkout_region(seed_index=s)
        rec = {"seed": s, "ok": active is not None}
        if active is not None:
            rec.update(ra=float(region.ra), dec=float(region.dec), radius=float(region.radius),
                       active=active["source_index"].tolist(),
                       fixed=[] if fixed is None else fixed["source_index"].tolist())
            held.append((active, fixed))
        out.append(rec)
        if k % 4 == 3 and held:
            a, f = held.pop(0)
            if circular:
                a = a.copy()
                a["q"] = np.clip(a["q"] * 1.01, 0, 0.99)
                a[bands[0]] *= 1.5
                sc.checkin_region(a, f, niter=3, taskID=k)
            else:
                sc.checkin_region(a, f, niter=1)
    return out


def _same_checkouts(mine, ref):
    assert len(mine) == len(ref)
    for m, r in zip(mine, ref):
        assert m["seed"] == r["seed"] and m["ok"] == r["ok"], (m, r)
        if r["ok"]:
            assert m["active"] == r["active"] and m["fixed"] == r["fixed"], (m["seed"], m, r)
            np.testing.assert_allclose([m["ra"], m["dec"], m["radius"]], [r["ra"], r["dec"], r["radius"]],
                                       rtol=1e-12, atol=1e-12)


def test_circular_checkouts_match_the_reference(gold):
    cat, bands = catalog(gold)
    sc = SS.SuperScene(sourcecat=cat, bands=bands, maxactive_per_patch=15, maxradius=6., boundary_radius=8.,
                       nscale=3, minradius=1)
    ref = gold["circular"]
    _same_checkouts(_run_checkouts(sc, bands, True), ref["checkouts"])
    for c, v in ref["state"].items():
        np.testing.assert_array_equal(sc.sourcecat[c], np.array(v, dtype=sc.sourcecat[c].dtype), err_msg=c)
    assert (sc.n_active, sc.n_fixed) == (ref["n_active"], ref["n_fixed"])
    bnd, cov = sc.bounds_and_covs(np.array([3, 8, 9]))
    assert list(cov.shape) == ref["bounds_and_covs_shape"]
    assert sc.patchlog and all(isinstance(v, list) for v in sc.sourcelog.values())


@pytest.mark.parametrize("strict", [False, True])
def test_linked_scenes_match_the_reference(gold, strict):
    cat, bands = catalog(gold)
    ref = gold["linked_strict" if strict else "linked"]
    sc = SS.LinkedSuperScene(sourcecat=cat, bands=bands, maxactive_per_patch=15, maxradius=6.,
                             boundary_radius=8., nscale=3, minradius=1, buffer=0.3, roi=cat["roi"], strict=strict)
    for s, members in ref["grow"].items():
        assert sc.grow_source(int(s)) == members, s
    np.testing.assert_array_equal(sc.make_group_catalog(), np.array(ref["groups"]))
    _same_checkouts(_run_checkouts(sc, bands, False), ref["checkouts"])
    for c, v in ref["state"].items():
        np.testing.assert_array_equal(sc.sourcecat[c], np.array(v, dtype=sc.sourcecat[c].dtype), err_msg=c)
    assert sc.overlap_circle(53.1, -27.8, 2.0)["source_index"].tolist() == ref["overlap_circle"]


def test_bounds_match_the_reference(gold):
    cat, bands = catalog(gold)
    ref = gold["bounds"]
    plain = SS.make_bounds(cat, bands)
    unc = np.zeros(len(cat), dtype=[(b, np.float64) for b in bands])
    for b in bands:
        unc[b] = ref["unc"][b]
    withunc = SS.make_bounds(cat, bands, unccat=unc, dpos=np.array([0.1, 0.05]))
    for mine, r in ((plain, ref["plain"]), (withunc, ref["withunc"])):
        assert list(mine.dtype.names) == list(r.keys())
        for c in mine.dtype.names:
            np.testing.assert_allclose(mine[c], np.array(r[c]), rtol=1e-15, atol=0, err_msg=c)
    lo, hi = SS.bounds_vectors(plain[:5], bands, reference_coordinates=[53.1, -27.8])
    np.testing.assert_allclose(lo, ref["vectors"][0], rtol=1e-15, atol=1e-18)
    np.testing.assert_allclose(hi, ref["vectors"][1], rtol=1e-15, atol=1e-18)
    fl = np.array(ref["flux_in"])
    for mine, r in ((SS.flux_bounds(fl.copy(), 5.0), ref["flux_bounds"]),
                    (SS.flux_bounds(fl.copy(), 5.0, precisions=np.array(ref["prec"])), ref["flux_bounds_prec"])):
        np.testing.assert_allclose(mine[0], r[0], rtol=1e-14)
        np.testing.assert_allclose(mine[1], r[1], rtol=1e-14)


def test_random_seeds_are_valid_sources_and_regions_never_share_an_active_source(gold):
    # fixed sources may be shared by regions checked out together (they are
    # only subtracted); an active source belongs to one region at a time
    cat, bands = catalog(gold)
    sc = SS.SuperScene(sourcecat=cat, bands=bands, maxactive_per_patch=15, rng=np.random.default_rng(8))
    taken = set()
    n_out = 0
    for _ in range(200):
        w = sc.seed_weight()
        assert np.all(w[sc.sourcecat["is_valid"] == 0] == 0) and abs(w.sum() - 1) < 1e-12
        region, active, fixed = sc.checkout_region()
        if active is None:
            continue
        ids = set(active["source_index"].tolist())
        assert not (ids & taken)
        taken |= ids
        n_out += 1
    assert n_out > 10
    assert sc.n_active == int(sc.sourcecat["is_active"].sum()) == len(taken)


def test_checkin_restores_availability_and_counts(gold):
    cat, bands = catalog(gold)
    sc = SS.LinkedSuperScene(sourcecat=cat, bands=bands, maxactive_per_patch=10, roi=cat["roi"], target_niter=2)
    region, active, fixed = sc.checkout_region(seed_index=0)
    assert sc.undone and sc.n_active == len(active)
    a = active.copy()
    a["rhalf"] = 0.2
    covs = np.tile(np.eye(len(sc.parameter_columns)) * 2, (len(a), 1, 1))
    sc.checkin_region(a, fixed, niter=2, block_covs=covs, taskID="t0")
    idx = a["source_index"]
    assert np.all(sc.sourcecat["rhalf"][idx] == 0.2) and np.all(sc.sourcecat["n_iter"][idx] == 2)
    assert np.all(sc.sourcecat["is_valid"] == 1) and sc.n_active == 0 and sc.n_fixed == 0
    assert np.all(sc.covariance_matrices[idx] == covs)
    assert sc.sourcelog[int(idx[0])] == ["t0"] and sc.patchlog == ["t0"]
    sc.reset()
    assert np.all(sc.sourcecat["n_iter"] == 0)


def test_state_file_and_catalog_roundtrip(tmp_path, gold):
    cat, bands = catalog(gold)
    path = str(tmp_path / "scene.fits")
    with SS.SuperScene(sourcecat=cat.copy(), bands=bands, statefile=path) as sc:
        sc.checkout_region(seed_index=5)
    back = F.read_fits(path)[1].data
    for c in ("ra", "dec", "is_active", "is_valid", bands[0]):
        np.testing.assert_array_equal(back[c], sc.sourcecat[c])
    assert os.path.exists(path.replace(".fits", "_log.json"))
    # a raw input catalog: FILTERS in the primary header, shapes clipped on the way in
    raw = np.zeros(4, dtype=[("ra", ">f8"), ("dec", ">f8"), ("q", ">f8"), ("pa", ">f8"), ("sersic", ">f8"),
                             ("rhalf", ">f8"), ("F200W", ">f8"), ("F444W", ">f8"), ("extra", ">f4")])
    raw["ra"], raw["dec"] = 53.1 + np.arange(4) * 1e-4, -27.8
    raw["q"], raw["pa"], raw["sersic"] = [0.1, 0.5, 0.9, 1.2], [-3, 0, 1, 3], [0.5, 2, 4, 6]
    raw["rhalf"], raw["F200W"], raw["F444W"] = [0.01, 0.1, 0.2, 0.5], 1.0, 2.0
    rp = str(tmp_path / "raw.fits")
    F.write_fits(rp, [({"FILTERS": "F200W, F444W"}, None), ({}, raw)])
    sc2, b2, hdr = SS.rectify_catalog(rp)
    assert b2 == ["F200W", "F444W"]
    np.testing.assert_allclose(sc2["q"], [0.2, 0.5, 0.9, 0.99])
    np.testing.assert_allclose(sc2["rhalf"], [0.051, 0.1, 0.2, 0.29])
    np.testing.assert_allclose(sc2["sersic"], [1.01, 2, 4, 4.99])
    np.testing.assert_allclose(sc2["pa"], [-2, 0, 1, 2])
    assert list(sc2["source_index"]) == [0, 1, 2, 3]
    raw["q"][0] = np.nan
    F.write_fits(rp, [({"FILTERS": "F200W, F444W"}, None), ({}, raw)])
    with pytest.raises(ValueError):
        SS.rectify_catalog(rp)


def test_pa_conversion_and_bound_checks():
    pa = SS.convert_pa(np.array([0.0, 2.0, -2.0, 4.5, np.pi / 2]))
    np.testing.assert_allclose(pa, [0.0, 2.0 - np.pi, -2.0 + np.pi, 4.5 - np.pi, np.pi / 2])
    np.testing.assert_allclose(SS.convert_pa(np.array([90.0 + 180.0]), from_deg=True), [np.pi / 2])
    np.testing.assert_allclose(SS.convert_pa(np.array([0.5, -0.5]), rotate=True), [0.5 - np.pi / 2, np.pi / 2 - 0.5])
    cat = np.zeros(2, dtype=SS.sourcecat_dtype(bands=["F200W"]))
    cat["ra"], cat["dec"], cat["q"], cat["pa"], cat["sersic"], cat["rhalf"], cat["F200W"] = \
        10.0, 1.0, 0.8, 0.1, 2.0, 0.1, 5.0
    b = SS.make_bounds(cat, ["F200W"])
    SS.check_bounds(cat, b)
    cat["q"][1] = 1.5
    with pytest.raises(AssertionError, match="'q'"):
        SS.check_bounds(cat, b)
    cat["q"][1] = 0.8
    act = cat.copy()
    act["F200W"] = [1e6, -1e6]
    SS.adjust_bounds(b, ["F200W"], None, active=act, minflux=-1.0, maxfluxfactor=0)
    assert np.all(act["F200W"] < b["F200W"][:, 1]) and np.all(act["F200W"] > b["F200W"][:, 0])
    assert np.all(b["F200W"][:, 0] <= -1.0)


def test_missing_columns_are_reported():
    bad = np.zeros(3, dtype=[("ra", float), ("dec", float)])
    with pytest.raises(ValueError, match="rhalf"):
        SS.SuperScene(sourcecat=bad, bands=[])
