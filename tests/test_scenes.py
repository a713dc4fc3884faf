"""Host side of scene handling: packing a scene's source metadata over a
patch's pixels, the catalog round trip, band splits and the one-band flux
solve (CPU; the device paths are in test_gpu_render.py)."""

import numpy as np

from forcepho_b200 import synthetic as S
from forcepho_b200.fitting import optimize_one_band
from forcepho_b200.sources import Scene


def _patch():
    return S.config_multiband(seed=21, n_sources=6, n_bands=3, exp_per_band=2, size=40)


def test_meta_for_reproduces_the_packed_scene():
    p = _patch()
    meta = p.meta_for(p.scene)
    assert meta["n_sources"] == p.n_sources
    for k in ("D", "CW", "crpix", "crval", "psfgauss", "psfgauss_start"):
        assert meta[k].tobytes() == np.asarray(getattr(p, k)).tobytes(), k


def test_subset_scene_meta_is_the_matching_slice():
    p = _patch()
    sub = Scene([p.scene.sources[i] for i in (1, 4)])
    meta = p.meta_for(sub)
    assert meta["n_sources"] == 2
    for k in ("D", "CW", "crpix", "crval"):
        np.testing.assert_array_equal(meta[k], np.asarray(getattr(p, k))[:, [1, 4]])
    # every source of an exposure reads the exposure's first PSF block
    npsf = p.n_psf_per_source[p.exposure_band()]
    for e in range(p.n_exp):
        a = meta["psfgauss"][meta["psfgauss_start"][e]:meta["psfgauss_start"][e] + npsf[e]]
        b = p.psfgauss[p.psfgauss_start[e]:p.psfgauss_start[e] + npsf[e]]
        assert a.tobytes() == b.tobytes()
    p.validate()


def test_catalog_round_trip_and_pack_meta():
    p = _patch()
    cat = p.catalog()
    scene = p.set_scene(cat)
    a, b = scene.get_proposal(), p.scene.get_proposal()
    assert a.tobytes() == b.tobytes()
    q = S.config_multiband(seed=21, n_sources=6, n_bands=3, exp_per_band=2, size=40)
    q.pack_meta(q.set_scene(cat[2:5]))
    assert q.n_sources == 3 and q.D.shape == (q.n_exp, 3, 2, 2)
    q.validate()


def test_split_band():
    p = _patch()
    parts = p.split_band("ierr")
    assert [len(x) for x in parts] == list(p.band_N_pix)
    np.testing.assert_array_equal(np.concatenate(parts), p.ierr)


def test_optimize_one_band_is_weighted_least_squares():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(5, 400))
    w = rng.uniform(0.5, 2.0, 400)
    f = rng.uniform(1, 10, 5)
    y = f @ X + rng.normal(0, 0.01, 400) / w
    flux, ATA = optimize_one_band(X, w, y)
    want = np.linalg.lstsq((X * w).T, y * w, rcond=None)[0]
    np.testing.assert_allclose(flux[:, 0], want, rtol=1e-10)
    np.testing.assert_allclose(ATA, (X * w) @ (X * w).T, rtol=1e-12)


def test_empty_scene_packs_and_validates():
    p = _patch()
    p.pack_meta(Scene([]))
    assert p.n_sources == 0 and p.D.shape == (p.n_exp, 0, 2, 2) and len(p.psfgauss) == 0
    assert p.validate()
