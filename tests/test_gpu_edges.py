"""Edge cases of the kernel limits (forcepho/src/kernel_limits.h): a patch with
MAXBANDS bands and MAXSOURCES sources at once, and a patch with no sources,
through both the tiled and the plain path, against the FP64 oracle and the
reference CPU kernel."""

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import (CHI2_F64, CHI2_REF, GRAD_F64, GRAD_REF, band_scales, chi2_err, chi2_raw_err, chi2_scale,
                        grad_err, ref_gap_explained)

pytestmark = pytest.mark.gpu


def _render(p, prop):
    return O.render(p, prop, precision="f64")


@pytest.mark.parametrize("kind", ["tiled", "plain"])
def test_max_bands_and_sources(kind):
    from forcepho_b200 import synthetic as S
    from forcepho_b200.kernel_limits import MAXBANDS, MAXSOURCES
    from forcepho_b200.proposal import B200Proposer, PlainProposer
    p = S.config_multiband(seed=50, render=_render, n_sources=MAXSOURCES, n_bands=MAXBANDS, exp_per_band=1,
                           size=20)
    p.return_residual = True
    p.send_to_device()
    prop = p.scene.get_proposal().copy()
    prop["q"] *= 0.97
    pr = B200Proposer() if kind == "tiled" else PlainProposer()
    chi2, dchi2, res = pr.evaluate_proposal(prop, patch=p, unpack=False)
    assert chi2.shape == (MAXBANDS,) and dchi2.shape == (MAXBANDS, MAXSOURCES, 7)
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
    scale = float(np.max(np.abs(r64)))
    assert np.max(np.abs(res.astype(np.float64) - r64)) <= 1e-5 * scale


@pytest.mark.parametrize("kind", ["tiled", "plain"])
def test_no_sources(kind):
    from forcepho_b200 import synthetic as S
    from forcepho_b200.proposal import B200Proposer, PlainProposer
    from forcepho_b200.structs import source_struct_dtype
    p = S.config_multiband(seed=51, n_sources=3, n_bands=2, exp_per_band=2, size=24)
    p.pack_meta(S.Scene([]))
    assert p.n_sources == 0
    p.return_residual = True
    p.send_to_device()
    pr = B200Proposer() if kind == "tiled" else PlainProposer()
    chi2, dchi2, res = pr.evaluate_proposal(np.zeros(0, dtype=source_struct_dtype), patch=p, unpack=False)
    # no model: residual = data, chi2 = sum (d ierr - d ierr)(d ierr + d ierr) = 0
    np.testing.assert_array_equal(chi2, np.zeros(p.n_bands))
    assert dchi2.shape == (p.n_bands, 0, 7)
    np.testing.assert_array_equal(res, p.data)
