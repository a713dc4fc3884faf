"""Size-independent properties of the batched evaluation, on patches drawn
from the bench's batched distribution (sources 1-30, bands 1-8, exposures 1-4
per band, up to 256x256 pixels per exposure), where the FP64 oracle would be
slow:

* flux homogeneity: the model is linear in the fluxes and the MAX_EXP_ARG
  cutoff does not depend on them, so for chi2 = sum (r^2 - d^2) ierr^2
  with r = d - model, chi2(2 f)[b] = 2 sum_s f_sb d chi2 / d f_sb at f, band
  by band;
* shift invariance: moving every pixel and every source by the same whole
  number of pixels leaves chi2 and the gradient unchanged (up to FP32
  rounding of the coordinates)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _patches(n=24, seed=4):
    from forcepho_b200 import synthetic as S
    shapes = S.batched_shapes(seed=seed, n_patches=512)
    rng = np.random.default_rng(77)
    out = []
    for i in sorted(rng.choice(512, n, replace=False)):
        sh = shapes[i]
        r = np.random.default_rng(sh["seed"])
        p = S.make_patch(r, n_sources=sh["n_sources"], exp_per_band=sh["exp_per_band"], exp_pix=sh["exp_pix"],
                         n_psf=4, source_params=S._broad_source, raster_width=256)
        S.add_noise(p, r, r.uniform(0.5, 2.0, p.n_exp))
        p.return_residual = False
        p.send_to_device()
        out.append(p)
    return out


@pytest.fixture(scope="module")
def batch():
    return _patches()


def _props(patches, scale=1.0):
    out = []
    for p in patches:
        q = p.scene.get_proposal().copy()
        q["q"] = np.clip(q["q"] * 0.97, 0.2, 0.99)
        q["fluxes"] = (q["fluxes"] * scale).astype(np.float32)
        out.append(q)
    return out


def test_flux_homogeneity_on_the_batched_distribution(batch):
    from forcepho_b200.batch import BatchedProposer
    bp = BatchedProposer(batch)
    res1 = bp.evaluate_proposals(_props(batch, 1.0))
    res2 = bp.evaluate_proposals(_props(batch, 2.0))
    worst = 0.0
    for p, prop, (c1, g1), (c2, _) in zip(batch, _props(batch), res1, res2):
        ns, nb = int(p.n_sources), p.n_bands
        f = np.asarray(prop["fluxes"][:, :nb], np.float64)          # [source, band]
        fg = np.einsum("sb,bs->b", f, np.asarray(g1[:, :, 0], np.float64))
        # chi2 terms scale with sum d^2 ierr^2 over the band; relative to
        # max(|chi2(2f)|, 1e-3 of that), as the raw chi2 tolerance does
        for b in range(nb):
            e0, ne = int(p.band_start[b]), int(p.band_N[b])
            s0 = int(p.exposure_start[e0])
            s1 = int(p.exposure_start[e0 + ne - 1] + p.exposure_N[e0 + ne - 1])
            dd = float(np.sum((p.data[s0:s1].astype(np.float64) * p.ierr[s0:s1]) ** 2))
            den = max(abs(c2[b]), 1e-3 * dd)
            worst = max(worst, abs(c2[b] - 2.0 * fg[b]) / den)
        assert ns > 0
    assert worst < 2e-5, worst


def test_shift_invariance(batch):
    from forcepho_b200.proposal import B200Proposer
    p = batch[0]
    prop = _props([p])[0]
    c0, g0 = B200Proposer().evaluate_proposal(prop, patch=p)
    p.free()
    saved = (p.xpix.copy(), p.ypix.copy(), p.crpix.copy())
    live = p.xpix >= 0
    try:
        p.xpix = np.where(live, p.xpix + 64, p.xpix).astype(np.float32)
        p.ypix = np.where(live, p.ypix + 32, p.ypix).astype(np.float32)
        p.crpix = (p.crpix + np.array([64.0, 32.0], np.float32)).astype(np.float32)
        p.send_to_device()
        c1, g1 = B200Proposer().evaluate_proposal(prop, patch=p)
    finally:
        p.xpix, p.ypix, p.crpix = saved
        p.send_to_device()
    from tolerances import grad_err
    assert np.max(np.abs(c1 - c0) / np.maximum(np.abs(c0), 1e-300)) < 1e-5
    assert grad_err(g1, g0) < 1e-4
