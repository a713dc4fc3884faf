"""Shape-space edges of the kernels against the FP64 oracle and the reference
CPU kernel: sources far outside the patch (every Gaussian culled: the model is
zero, chi2 = sum (d ierr - d ierr)(d ierr + d ierr) = 0 exactly, the gradient
zero) and extreme shapes (axis ratio 0.21, half-light radii from 0.03" to
0.6", Sersic indices at both ends of the amplitude table), and chunk tails of
every size in the adjoint."""

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import (CHI2_F64, CHI2_REF, GRAD_F64, GRAD_REF, band_scales, chi2_err, chi2_raw_err, chi2_scale,
                        grad_err, ref_gap_explained)

pytestmark = pytest.mark.gpu


def _patch(seed):
    from forcepho_b200 import synthetic as S
    p = S.config_multiband(seed=seed, render=lambda pp, pr: O.render(pp, pr, precision="f64"), n_sources=4,
                           n_bands=2, exp_per_band=2, size=48)
    p.return_residual = True
    p.send_to_device()
    return p


@pytest.mark.parametrize("kind", ["tiled", "plain"])
def test_sources_far_outside_the_patch(kind):
    from forcepho_b200.proposal import B200Proposer, PlainProposer
    p = _patch(80)
    prop = p.scene.get_proposal().copy()
    prop["ra"] += 1.0                      # one degree away: E >> MAX_EXP_ARG at every pixel
    prop["dec"] -= 1.0
    pr = B200Proposer() if kind == "tiled" else PlainProposer()
    chi2, dchi2, res = pr.evaluate_proposal(prop, patch=p, unpack=False)
    np.testing.assert_array_equal(chi2, np.zeros(p.n_bands))
    np.testing.assert_array_equal(dchi2, np.zeros_like(dchi2))
    np.testing.assert_array_equal(res, p.data)
    c64, g64, _ = O.evaluate(p, prop, precision="f64", return_residual=True)
    np.testing.assert_array_equal(c64, np.zeros(p.n_bands))


@pytest.mark.parametrize("kind", ["tiled", "plain"])
@pytest.mark.parametrize("shape", [dict(q=0.21, rhalf=0.2, sersic=2.0), dict(q=0.9, rhalf=0.03, sersic=1.0),
                                   dict(q=0.5, rhalf=0.6, sersic=6.0), dict(q=0.35, rhalf=0.1, sersic=0.85)])
def test_extreme_shapes(kind, shape):
    from forcepho_b200.proposal import B200Proposer, PlainProposer
    p = _patch(81)
    for g in p.scene.sources:
        g.q, g.rhalf, g.sersic = shape["q"], shape["rhalf"], shape["sersic"]
        g.pa = 0.7
    prop = p.scene.get_proposal().copy()
    pr = B200Proposer() if kind == "tiled" else PlainProposer()
    chi2, dchi2, res = pr.evaluate_proposal(prop, patch=p, unpack=False)
    c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    cr, gr, _ = O.ref_evaluate(p, prop)
    sc = chi2_scale(chi2, p.data, p.ierr, r64)
    assert chi2_err(chi2, cr, sc) < CHI2_REF
    assert grad_err(dchi2, gr) < GRAD_REF
    tol_c, tol_g = (CHI2_F64, GRAD_F64) if kind == "tiled" else (CHI2_REF, GRAD_REF)
    assert chi2_err(chi2, c64, sc) < tol_c
    assert chi2_raw_err(chi2, c64, band_scales(p, r64)) < tol_c
    assert ref_gap_explained(chi2, cr, c64, tol_c, band_scales(p, r64))
    assert grad_err(dchi2, g64) < tol_g


@pytest.mark.parametrize("n_sources", [1, 2, 3, 4])
def test_partial_groups_of_every_size(n_sources):
    """1-Gaussian PSFs (9 image Gaussians per source) on 256-pixel tiles: over
    these four patches the tiles keep 2 to 30 Gaussians in their last group,
    so the adjoint replicates it 1, 2, 3, 4, 5, 6 and 8 times.  Tiled results
    match the FP64 oracle."""
    from forcepho_b200 import synthetic as S
    from forcepho_b200.proposal import B200Proposer
    p = S.config_multiband(seed=90 + n_sources, render=lambda pp, pr: O.render(pp, pr, precision="f64"),
                           n_sources=n_sources, n_bands=2, exp_per_band=1, size=64, n_psf=1)
    p.return_residual = True
    p.send_to_device()
    prop = p.scene.get_proposal().copy()
    prop["q"] = np.clip(prop["q"] * 0.97, 0.2, 0.99)
    chi2, dchi2, res = B200Proposer(tile_pixels=256).evaluate_proposal(prop, patch=p, unpack=False)
    c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    sc = chi2_scale(chi2, p.data, p.ierr, r64)
    assert chi2_err(chi2, c64, sc) < CHI2_F64
    assert chi2_raw_err(chi2, c64, band_scales(p, r64)) < CHI2_F64
    assert grad_err(dchi2, g64) < GRAD_F64
