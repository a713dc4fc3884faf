"""The dispatcher's GPU work unit end to end: a field of sources in a FITS
image set, a SuperScene over their catalog, rounds of regions packed from the
images, fixed sources subtracted on the device, fluxes solved, and chi2 and
gradients of each round's patches from one batched launch, checked against
the FP64 oracle on the same packed patches."""

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import CHI2_F64, GRAD_F64, band_scales, chi2_raw_err, grad_err

pytestmark = pytest.mark.gpu

BANDS = ["B0", "B1"]


def _field(rng, n=12):
    from forcepho_b200 import superscene as SS
    cat = np.zeros(n, dtype=SS.sourcecat_dtype(bands=BANDS))
    # within the 120 x 96 pixel (3.6" x 2.9") images around (53.1, -27.8)
    dx, dy = rng.uniform(-1.4, 1.4, n), rng.uniform(-1.1, 1.1, n)
    cat["ra"] = 53.1 + dx / 3600. / np.cos(np.deg2rad(-27.8))
    cat["dec"] = -27.8 + dy / 3600.
    cat["q"], cat["pa"] = rng.uniform(0.5, 0.9, n), rng.uniform(-1, 1, n)
    cat["sersic"], cat["rhalf"] = rng.uniform(1.2, 3.5, n), rng.uniform(0.05, 0.12, n)
    cat["roi"] = 3 * cat["rhalf"]
    for b in BANDS:
        cat[b] = rng.uniform(100, 300, n)
    return cat


def _truth_patcher(paths, truth):
    from test_stores import _PSF
    from forcepho_b200.stores.patch import FITSPatch

    class TruthPatch(FITSPatch):
        """Image noise plus the FP64 model of every true source."""

        def build_patch(self, region=None, sourcecat=None, allbands=BANDS, tweak_background=False):
            super().build_patch(region, None, allbands=allbands)
            scene = self.set_scene(truth)
            self.pack_meta(scene)
            self.data = (self.data + O.render(self, scene.get_proposal())).astype(np.float32)
            if sourcecat is not None:
                self.pack_meta(self.set_scene(sourcecat))

    def make_patcher():
        p = TruthPatch(fitsfiles=paths)
        p.psfstore = _PSF()
        return p

    return make_patcher


def test_hmc_rounds_on_a_fits_field(tmp_path):
    """The sampling work unit: every region of a round sampled together on
    the device within its prior bounds; the truth lies within the posterior
    (fluxes within a few posterior standard deviations of the posterior
    means; shapes are free, so the flux posterior is wide where flux and size
    trade off) and the scene counts the draws."""
    from test_stores import make_image_set
    from forcepho_b200 import dispatcher as D
    from forcepho_b200 import superscene as SS

    rng = np.random.default_rng(43)
    paths = make_image_set(tmp_path, seed=11, size=(120, 96))
    truth = _field(rng)
    # the catalog starts at the truth: fixed sources are then subtracted
    # exactly, and the posterior of the active ones must contain the truth
    cat = truth.copy()
    start = cat.copy()
    scene = SS.SuperScene(sourcecat=cat, bands=BANDS, maxactive_per_patch=4, maxradius=0.6, boundary_radius=0.8,
                          nscale=3, minradius=0.15, target_niter=40, maxactive_fraction=0.9,
                          rng=np.random.default_rng(6))
    # narrow shape priors around the truth: the flux posterior is then nearly
    # Gaussian and 40 draws sample it well (with free shapes, flux and size
    # trade off and a short chain understates the width along that direction)
    bc = scene.bounds_catalog
    for c, h in (("q", 0.02), ("pa", 0.05), ("sersic", 0.05), ("rhalf", 0.005)):
        bc[c][:, 0] = truth[c] - h
        bc[c][:, 1] = truth[c] + h
    results = []
    work = D.hmc_work(_truth_patcher(paths, truth), BANDS, n_warmup=40, n_draws=40, n_steps=8, seed=3,
                      tile_pixels=256)

    def logged(tasks):
        res = work(tasks)
        for t, r in zip(tasks, res):
            r["ids"] = t["active"]["source_index"].copy()
        results.extend(res)
        return res

    rounds = D.run(scene, logged, batch_per_rank=4, max_rounds=2)
    assert rounds and len(results) == sum(r["tasks"] for r in rounds)
    for r in results:
        assert 0.2 < r["acceptance"] <= 1.0, r["acceptance"]
        for c in BANDS + ["ra", "dec", "q", "pa", "sersic", "rhalf"]:
            assert np.all(np.isfinite(r["final"][c]))
        if r["covs"] is not None:
            assert r["covs"].shape == (len(r["final"]), 8, 8)
            assert np.all(np.linalg.eigvalsh(r["covs"]) > -1e-12)
    done = scene.sourcecat["n_iter"] >= 40
    assert done.sum() >= 2
    SS.check_bounds(scene.sourcecat[done], scene.bounds_catalog[done])
    z = []
    for r in results:
        assert r["covs"] is not None
        sd = np.sqrt(np.diagonal(r["covs"], axis1=1, axis2=2))
        for k, i in enumerate(r["ids"]):
            for j, b in enumerate(BANDS):
                z.append(abs(r["final"][b][k] - truth[b][i]) / sd[k, j])
    z = np.array(z)
    assert np.all(z < 5) and np.median(z) < 2.0, z
    assert not np.array_equal(scene.sourcecat[BANDS[0]][done], start[BANDS[0]][done])


def test_flux_fit_rounds_on_a_fits_field(tmp_path):
    from test_stores import make_image_set
    from forcepho_b200 import dispatcher as D
    from forcepho_b200 import superscene as SS
    from forcepho_b200.proposal import B200Proposer

    rng = np.random.default_rng(41)
    paths = make_image_set(tmp_path, seed=9, size=(120, 96))
    truth = _field(rng)

    make_patcher = _truth_patcher(paths, truth)
    cat = truth.copy()
    for b in BANDS:
        cat[b] *= rng.uniform(0.7, 1.3, len(cat))       # starting fluxes off the truth
    start = cat.copy()                                  # the scene updates cat in place
    scene = SS.SuperScene(sourcecat=cat, bands=BANDS, maxactive_per_patch=4, maxradius=0.6, boundary_radius=0.8,
                          nscale=3, minradius=0.15, target_niter=1, maxactive_fraction=0.9,
                          rng=np.random.default_rng(5))
    work = D.flux_fit_work(make_patcher, BANDS, keep_patches=True)
    checked = []

    def checked_work(tasks):
        res = work(tasks)
        for t, r in zip(tasks, res):
            p = r.pop("patch")
            prop = p.scene.get_proposal()
            c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
            assert chi2_raw_err(r["chi2"], c64, band_scales(p, r64)) < CHI2_F64
            # at the fitted fluxes, near the likelihood's mode, the gradient
            # columns cancel between pixels while each pair's rounding stays;
            # the gradients are compared off the mode, as in every parity test
            off = prop.copy()
            off["fluxes"] *= 1.05
            off["q"] = np.clip(off["q"] * 0.95, 0.2, 0.99)
            # about 5 pixels: the FP32 pixel coordinates and Gaussian centres
            # (rounding up to 4e-6 px at x ~ 100) move chi2 and its position
            # gradient by that much; far from the mode it is small beside them
            off["ra"] += 4e-5
            off["dec"] -= 4e-5
            c, g = B200Proposer().evaluate_proposal(off, patch=p)[:2]
            c64, g64, r64 = O.evaluate(p, off, precision="f64", return_residual=True)
            assert chi2_raw_err(c, c64, band_scales(p, r64)) < CHI2_F64
            assert grad_err(g, g64) < GRAD_F64
            checked.append(t["taskid"])
            p.free()
        return res

    rounds = D.run(scene, checked_work, batch_per_rank=4, max_rounds=20)
    assert len(checked) == sum(r["tasks"] for r in rounds) > 0
    done = scene.sourcecat["n_iter"] >= 1
    assert done.sum() >= len(cat) // 2
    # fitted fluxes sit closer to the truth than the starting ones
    for b in BANDS:
        err0 = np.abs(start[b][done] - truth[b][done])
        err1 = np.abs(scene.sourcecat[b][done] - truth[b][done])
        assert np.median(err1) < np.median(err0)
