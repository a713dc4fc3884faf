"""Sampling bounds of the device HMC: the RA range of a source is 0.3 arcsec
divided by cos(dec) at that source, read from the patch's own astrometry
(CW = 3600 D diag(cos dec, 1)), whatever the field's declination."""

import numpy as np
import pytest


@pytest.mark.parametrize("dec0", [-27.8, 0.0, 62.2])
def test_ra_bound_follows_the_patch_declination(monkeypatch, dec0):
    from forcepho_b200 import synthetic as S
    from forcepho_b200.hmc import default_bounds, source_cos_dec
    monkeypatch.setattr(S, "REF_COORD", np.array([53.1, dec0]))
    p = S.config_multiband(seed=7, n_sources=3, n_bands=2, exp_per_band=2, size=32)
    ns, nb = int(p.n_sources), p.n_bands
    want = np.cos(np.deg2rad(dec0 + np.array([g.dec for g in p.scene.sources])))
    np.testing.assert_allclose(source_cos_dec(p, ns), want, rtol=1e-6)
    th = p.scene.get_all_source_params()
    lo, hi = default_bounds(p, th)
    per = nb + 6
    half_ra = (hi - lo).reshape(ns, per)[:, nb] / 2
    half_dec = (hi - lo).reshape(ns, per)[:, nb + 1] / 2
    np.testing.assert_allclose(half_dec, 0.3 / 3600, rtol=1e-12)
    np.testing.assert_allclose(half_ra * want, 0.3 / 3600, rtol=1e-6)
