"""Precision at detector-scale pixel coordinates.

forcepho's exposures carry absolute detector pixel coordinates (thousands of
pixels), where an FP32 coordinate is only good to 1e-4 px.  The tiled kernels
work in coordinates relative to each tile's origin, with the Gaussian centre
rebuilt there from its FP32 value and rounding residual, so the model keeps
its precision: the raw chi2 and gradient bounds against the FP64 oracle hold
for the same scene placed at (2000, 1500) as at the origin.  (Rounding the
centre alone to FP32 at these coordinates moves chi2 by up to 1.5e-5 of
itself on these patches.)"""

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import CHI2_F64, GRAD_F64, band_scales, chi2_raw_err, grad_err

pytestmark = pytest.mark.gpu


def _bright(rng, nb):
    return dict(flux=rng.uniform(100, 300, nb), q=rng.uniform(0.5, 0.9), pa=rng.uniform(-1, 1),
                sersic=rng.uniform(1.2, 3.5), rhalf=rng.uniform(0.05, 0.12))


def _patch(seed, offset):
    from forcepho_b200 import synthetic as S
    rng = np.random.default_rng(seed)
    p = S.make_patch(rng, n_sources=3, exp_per_band=[2, 1], exp_pix=[(120, 96)] * 3, n_psf=4,
                     source_params=_bright)
    p.xpix[:] += offset[0]
    p.ypix[:] += offset[1]
    p.crpix[..., 0] += offset[0]
    p.crpix[..., 1] += offset[1]
    truth = p.scene.get_proposal()
    p.data[:] = (O.render(p, truth) + rng.normal(0, 1, p.npix)).astype(np.float32)
    p.ierr[:] = 1.0
    prop = truth.copy()
    prop["ra"] += 1e-5                       # about a pixel off the truth
    prop["dec"] -= 1e-5
    prop["q"] = np.clip(prop["q"] * 0.95, 0.2, 0.99)
    return p, prop


@pytest.mark.parametrize("offset", [(0.0, 0.0), (2000.0, 1500.0), (7000.0, 6000.0)])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_bright_scene_far_from_the_origin(seed, offset):
    from forcepho_b200.proposal import B200Proposer
    p, prop = _patch(seed, offset)
    p.return_residual = False
    p.send_to_device()
    chi2, dchi2 = B200Proposer().evaluate_proposal(prop, patch=p)
    c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    assert chi2_raw_err(chi2, c64, band_scales(p, r64)) < CHI2_F64
    assert grad_err(dchi2, g64) < GRAD_F64


def test_census_in_tile_coordinates():
    """The pair census evaluates the same tile-relative exponent: no pair
    within the cutoff belongs to a culled Gaussian, far from the origin too."""
    from forcepho_b200.batch import BatchedProposer
    patches = [_patch(s, (7000.0, 6000.0))[0] for s in (3, 4)]
    for p in patches:
        p.return_residual = False
        p.send_to_device()
    bp = BatchedProposer(patches, tile_pixels=256, use_graph=False)
    bp.set_proposals_async([p.scene.get_proposal() for p in patches])
    evaluated, active, dropped = bp.count_pairs()
    assert dropped == 0 and 0 < active <= evaluated
