"""Patch packing from image stores (forcepho_b200.stores), on the CPU:

* the FITS reader and writer, the TAN WCS, the HDF5 reader;
* the reference's own test image set (tests/data/test_image) packed by
  FITSPatch: the packed arrays equal the committed fixture bit for bit, and
  the catalog's model leaves residuals at the noise level (the packing, WCS
  and PSF store reproduce the reference's simulated image);
* a multi-band, multi-exposure FITS image set written here, packed and
  rendered by the FP64 oracle;
* StorePatch over a super-pixel store and a JSON header store;
* PatchFarm work lists over packed patches.
Tests that read the reference's files skip where they are absent."""

import json
import os

import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O

REF_ROOT = O.reference_root()
IMAGE = os.path.join(REF_ROOT, "tests", "data", "test_image", "sersic1.0_rhalf0.150_snr050_noise1_data.fits")
PSF = os.path.join(REF_ROOT, "tests", "data", "test_image", "sersic1.0_rhalf0.150_snr050_noise1_psf.h5")
SPLINES = os.path.join(REF_ROOT, "tests", "data", "sersic_splinedata_large.h5")
needs_reference = pytest.mark.skipif(not os.path.exists(IMAGE), reason="reference test data absent")


def test_fits_round_trip(tmp_path):
    from forcepho_b200.stores import fits as F
    img = np.arange(12, dtype=np.float32).reshape(3, 4) * 0.5
    img64 = np.linspace(-1, 1, 20).reshape(4, 5)
    ints = np.arange(6, dtype=np.int16).reshape(2, 3)
    tab = np.zeros(3, dtype=[("id", np.int32), ("ra", np.float64), ("flux", np.float32, (2,)), ("name", "S5")])
    tab["id"] = [1, 2, 3]
    tab["ra"] = [53.1, 53.2, 53.3]
    tab["flux"] = [[1, 2], [3, 4], [5, 6]]
    tab["name"] = [b"a", b"bb", b"ccc"]
    path = str(tmp_path / "t.fits")
    F.write_fits(path, [({"FILTER": "F200W", "CRPIX1": 1.5, "NOTE": "it's", "FLAG": False}, img),
                        ({"EXTNAME": "ERR"}, img64), ({}, ints), ({"FILTERS": "A,B"}, tab)])
    h = F.read_fits(path)
    assert len(h) == 4
    assert h[0].header["FILTER"] == "F200W" and h[0].header["CRPIX1"] == 1.5
    assert h[0].header["NOTE"] == "it's" and h[0].header["FLAG"] is False
    assert np.array_equal(h[0].data, img) and h[0].data.dtype == np.float32
    assert np.array_equal(h[1].data, img64) and np.array_equal(h[2].data, ints)
    t = h[3].data
    assert h[3].header["FILTERS"] == "A,B"
    assert np.array_equal(t["id"], tab["id"]) and np.array_equal(t["ra"], tab["ra"])
    assert np.array_equal(t["flux"], tab["flux"]) and list(t["name"]) == [b"a", b"bb", b"ccc"]


def test_fits_card_values():
    from forcepho_b200.stores.fits import _value
    assert _value(" 'RA---TAN'           / comment") == "RA---TAN"
    assert _value(" 'O''HARA '") == "O'HARA"
    assert _value("                    T / yes") is True
    assert _value("                   42") == 42
    assert _value("  8.3333333333333E-06 / x") == 8.3333333333333e-06
    assert _value("  1.5D+02") == 150.0


def _tan_header(crval=(53.0, -27.0), crpix=(50.5, 50.5), cd=((-8.3333e-6, 0.0), (0.0, 8.3333e-6))):
    return {"CTYPE1": "RA---TAN", "CTYPE2": "DEC--TAN", "CRVAL1": crval[0], "CRVAL2": crval[1],
            "CRPIX1": crpix[0], "CRPIX2": crpix[1], "CD1_1": cd[0][0], "CD1_2": cd[0][1],
            "CD2_1": cd[1][0], "CD2_2": cd[1][1]}


def test_tan_wcs_known_answers_and_round_trips():
    from forcepho_b200.stores.wcs import TanWCS, scale_at_sky
    w = TanWCS(_tan_header(cd=((8.3333333333333e-6, 0), (0, 8.3333333333333e-6))))
    # the tangent point is CRPIX (FITS, 1-based), i.e. CRPIX - 1 at origin 0
    x, y = w.all_world2pix(53.0, -27.0, 0)
    assert abs(x - 49.5) < 1e-9 and abs(y - 49.5) < 1e-9
    # one arcsecond north of the tangent point: tan(1") / scale pixels along +y
    x, y = w.all_world2pix(53.0, -27.0 + 1 / 3600.0, 1)
    assert abs(x - 50.5) < 1e-9
    assert abs(y - 50.5 - np.rad2deg(np.tan(np.deg2rad(1 / 3600.0))) / 8.3333333333333e-6) < 1e-6
    # rotated, sheared CD at high declination: world -> pixel -> world
    w2 = TanWCS(_tan_header(crval=(210.0, 80.0), cd=((-5e-6, 3e-6), (2e-6, 6e-6))))
    px = np.array([0.0, 49.5, 99.0, 1e4, -3e3])
    py = np.array([0.0, 49.5, 10.0, -3e3, 2e3])
    ra, dec = w2.all_pix2world(px, py, 0)
    bx, by = w2.all_world2pix(ra, dec, 0)
    assert np.max(np.abs(bx - px)) < 1e-6 and np.max(np.abs(by - py)) < 1e-6
    CW, D = scale_at_sky((210.0, 80.0), w2)
    assert np.allclose(D, np.linalg.inv(w2.cd * 3600.0))
    assert np.allclose(CW, D * 3600.0 @ np.diag([np.cos(np.deg2rad(80.0)), 1.0]))
    with pytest.raises(ValueError):
        TanWCS(dict(_tan_header(), A_ORDER=2))


@needs_reference
def test_h5_reader_on_the_reference_stores():
    from forcepho_b200.splines import default_splines  # noqa: F401
    from forcepho_b200.stores.h5lite import H5File
    from forcepho_b200.stores.patch import PSFStore
    f = H5File(SPLINES)
    npz = np.load(os.path.join(os.path.dirname(O.HERE), "forcepho_b200", "data", "sersic_splinedata_large.npz"))
    for k in ("amplitudes", "nsersic", "rh", "radii"):
        assert np.array_equal(f[k].read(), npz[k])
    ps = PSFStore(PSF)
    assert ps.n_psf_per_source("CLEAR") == 9
    rows = ps.get_local_psf("CLEAR")
    assert len(rows) == 9 and np.array_equal(rows["sersic_bin"], np.arange(9))
    assert np.allclose(rows["Cxx"], 6.25) and np.allclose(rows["amp"], 1.0)


@needs_reference
def test_reference_image_set_packs_to_the_fixture_and_fits_its_noise():
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from golden.make_store_golden import ARRAYS, pack
    g = load_golden("fits_store.npz")
    p, region, cat = pack(IMAGE, PSF)
    for n in ARRAYS:
        assert np.array_equal(getattr(p, n), g[n]), n
    assert np.array_equal(p.patch_reference_coordinates, g["reference_coordinates"])
    p.validate()
    # the catalog model leaves residuals at the noise level of the image
    c, _, r = O.evaluate(p, p.scene.get_proposal(), precision="f64", return_residual=True)
    live = p.ierr > 0
    red = float(np.mean((r[live] * p.ierr[live]) ** 2))
    assert 0.85 < red < 1.15, red


def _patch_from_fixture(g):
    from conftest import patch_from_golden
    return patch_from_golden(g)


def test_fixture_patch_reproduces_its_oracle_outputs():
    g = load_golden("fits_store.npz")
    p = _patch_from_fixture(g)
    p.validate()
    for k in (0, 1):
        c, dc, _ = O.evaluate(p, g["proposal_%d" % k], precision="f64")
        assert np.array_equal(c, g["f64_chi2_%d" % k]) and np.array_equal(dc, g["f64_dchi2_%d" % k])


def make_image_set(tmp_path, seed=3, n_exp=(2, 1), size=(60, 48)):
    """FITS files of two bands (n_exp exposures each), a rotated TAN WCS per
    exposure, noise images with a few masked pixels in the uncertainty
    extension.  Models come from the oracle in the tests."""
    from forcepho_b200.stores import fits as F
    rng = np.random.default_rng(seed)
    paths = []
    for b, ne in enumerate(n_exp):
        for e in range(ne):
            t = rng.uniform(-0.3, 0.3)
            sc = 0.03 / 3600.0 * rng.uniform(0.95, 1.05)
            cd = sc * np.array([[-np.cos(t), np.sin(t)], [np.sin(t), np.cos(t)]])
            hdr = _tan_header(crval=(53.1 + rng.normal(0, 1e-5), -27.8 + rng.normal(0, 1e-5)),
                              crpix=(size[0] / 2 + 0.5, size[1] / 2 + 0.5), cd=cd)
            hdr["FILTER"] = "B%d" % b
            img = rng.normal(0, 1.0, (size[1], size[0])).astype(np.float32)
            unc = np.full_like(img, 1.0)
            unc[0, :5] = np.nan                          # masked pixels
            path = str(tmp_path / ("b%d_e%d.fits" % (b, e)))
            F.write_fits(path, [(hdr, img), ({}, unc)])
            paths.append(path)
    return paths


class _PSF:
    """A one-Gaussian-per-radius PSF store stand-in (the reference's test PSF shape)."""

    def n_psf_per_source(self, band):
        return 9

    def get_local_psf(self, band, source=None, wcs=None):
        from forcepho_b200.structs import psf_dtype
        out = np.zeros(9, dtype=psf_dtype)
        out["amp"] = 1.0
        out["Cxx"] = out["Cyy"] = 2.0 + 0.5 * (len(band) % 3)
        out["sersic_bin"] = np.arange(9)
        return out


def test_synthetic_image_set_packs_band_by_band(tmp_path):
    from forcepho_b200.stores.patch import FITSPatch
    from forcepho_b200.stores.region import CircularRegion
    paths = make_image_set(tmp_path)
    p = FITSPatch(fitsfiles=paths)
    p.psfstore = _PSF()
    cat = np.zeros(2, dtype=[(c, np.float64) for c in ("ra", "dec", "q", "pa", "sersic", "rhalf", "B0", "B1")])
    cat["ra"] = [53.1, 53.1 + 5e-5]
    cat["dec"] = [-27.8, -27.8 - 3e-5]
    cat["q"], cat["pa"], cat["sersic"], cat["rhalf"] = [0.8, 0.6], [0.3, -0.5], [2.0, 1.5], [0.1, 0.2]
    cat["B0"], cat["B1"] = [10.0, 5.0], [7.0, 3.0]
    region = CircularRegion(53.1, -27.8, 0.6 / 3600.0)
    p.build_patch(region, cat, allbands=["B0", "B1"])
    p.validate()
    assert p.n_bands == 2 and list(p.band_N) == [2, 1] and p.n_exp == 3 and p.n_sources == 2
    assert np.all(p.exposure_N % 64 == 0) and p.npix == int(np.sum(p.exposure_N))
    # masked and pad pixels carry no weight; pad pixels sit at (-1, -1)
    assert np.all(p.ierr[p.xpix < 0] == 0)
    # every exposure's sources land where its own WCS puts them
    for e, w in enumerate(p.wcses):
        for i in range(2):
            x, y = w.all_world2pix(cat["ra"][i], cat["dec"][i], 0)
            assert np.allclose(p.crpix[e, i], [x, y], atol=1e-3)
    assert np.allclose(p.crval[:, :, 0] + p.patch_reference_coordinates[0], cat["ra"][None, :])
    # the model peaks at the brighter source's position in each exposure
    m = O.render(p, p.scene.get_proposal())
    for e in range(p.n_exp):
        s0, n = int(p.exposure_start[e]), int(p.exposure_N[e])
        k = s0 + int(np.argmax(m[s0:s0 + n]))
        assert np.hypot(p.xpix[k] - p.crpix[e, 0, 0], p.ypix[k] - p.crpix[e, 0, 1]) < 1.5


def test_store_patch_over_a_superpixel_store(tmp_path):
    """StorePatch: exposures from the header store that overlap the region,
    the super-pixels with a corner inside it, in super-pixel order."""
    from forcepho_b200.stores import patch as SP
    from forcepho_b200.stores.region import CircularRegion
    nside, s = 64, 8
    rng = np.random.default_rng(1)
    images = {}
    headers = {}
    for band, exps in (("F200W", ["e1", "e2"]), ("F444W", ["e3"])):
        headers[band] = {}
        for ex in exps:
            h = _tan_header(crval=(53.1, -27.8), crpix=(32.5 + rng.normal(0, 2), 32.5),
                            cd=((-0.03 / 3600, 0), (0, 0.03 / 3600)))
            cards = "".join(("%-8s= %20s" % (k, ("'%s'" % v) if isinstance(v, str) else repr(v))).ljust(80)
                            for k, v in h.items()) + "END".ljust(80)
            headers[band][ex] = cards
            im = rng.normal(0, 1, (nside, nside)).astype(np.float32)
            images["%s/%s" % (band, ex)] = (im, np.ones_like(im))
    meta = str(tmp_path / "meta.json")
    with open(meta, "w") as f:
        json.dump(headers, f)

    class MemStore(SP.PixelStore):
        def __init__(self):
            self.nside_full = np.array([nside, nside])
            self.super_pixel_size = s
            self.xpix, self.ypix = self.pixel_coordinates()

        def data(self, epath):
            return self.superpixelize(*images[epath])

    p = SP.StorePatch.__new__(SP.StorePatch)
    SP.StorePatchBase.__init__(p)
    p.psfstore = _PSF()
    p.metastore = SP.MetaStore(meta)
    p.pixelstore = MemStore()
    region = CircularRegion(53.1, -27.8, 0.2 / 3600.0)
    cat = np.zeros(1, dtype=[(c, np.float64) for c in ("ra", "dec", "q", "pa", "sersic", "rhalf", "F200W", "F444W")])
    cat["ra"], cat["dec"], cat["q"], cat["sersic"], cat["rhalf"] = 53.1, -27.8, 0.7, 2.0, 0.1
    cat["F200W"], cat["F444W"] = 3.0, 4.0
    p.build_patch(region, cat, allbands=["F200W", "F444W"])
    p.validate()
    assert list(p.band_N) == [2, 1] and np.all(p.exposure_N % (s * s) == 0)
    # the packed pixels are exactly the image values at their coordinates
    for e, ep in enumerate(p.epaths):
        s0, n = int(p.exposure_start[e]), int(p.exposure_N[e])
        im = images[ep][0]
        xs, ys = p.xpix[s0:s0 + n].astype(int), p.ypix[s0:s0 + n].astype(int)
        assert np.array_equal(p.data[s0:s0 + n], im[xs, ys])
        # every super-pixel whose corner is within the region is in, and only those
        w = p.wcses[e]
        xc, yc = w.all_world2pix(53.1, -27.8, 0)
        d = np.hypot(xs - xc, ys - yc)
        assert d.min() < 8.0 and d.max() < 8.0 + 2 * s * 1.5


def test_patch_farm_work_lists_from_packed_patches(tmp_path):
    from forcepho_b200.distributed import balance
    from forcepho_b200.stores.patch import FITSPatch
    from forcepho_b200.stores.region import CircularRegion
    paths = make_image_set(tmp_path, seed=5)
    patches = []
    for k, r in enumerate((0.3, 0.5, 0.8, 0.4)):
        p = FITSPatch(fitsfiles=paths)
        p.psfstore = _PSF()
        cat = np.zeros(1 + k % 2, dtype=[(c, np.float64) for c in ("ra", "dec", "q", "pa", "sersic", "rhalf",
                                                                    "B0", "B1")])
        cat["ra"], cat["dec"], cat["q"], cat["sersic"], cat["rhalf"], cat["B0"], cat["B1"] = \
            53.1, -27.8, 0.7, 2.0, 0.1, 1.0, 1.0
        p.build_patch(CircularRegion(53.1, -27.8, r / 3600.0), cat, allbands=["B0", "B1"])
        patches.append(p)
    w = [p.n_pairs() for p in patches]
    lists = balance(w, 2)
    assert sorted(lists[0] + lists[1]) == [0, 1, 2, 3]
    loads = [sum(w[i] for i in l) for l in lists]
    assert max(loads) <= sum(w) - min(loads) and max(loads) >= sum(w) / 2
