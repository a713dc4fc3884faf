"""Store-packed patches on the GPU: the reference's own test image set, packed
by FITSPatch (committed fixture, so no reference files are read here),
evaluated by the tiled kernels against the FP64 oracle and the reference CPU
kernel outputs stored with it, the data/residual swap of tests/cswap_test.py
on it; and a multi-band FITS image set written and packed here, evaluated in
one batched pass with synthetic patches."""

import numpy as np
import pytest

from conftest import load_golden, patch_from_golden
from oracle import oracle as O
from tolerances import CHI2_F64, GRAD_F64, band_scales, chi2_raw_err, grad_err, ref_gap_explained

pytestmark = pytest.mark.gpu


def _fixture_patch():
    from forcepho_b200.synthetic import SyntheticPatch
    g = load_golden("fits_store.npz")
    return g, patch_from_golden(g, SyntheticPatch)


def test_reference_image_patch_on_the_gpu():
    from forcepho_b200.proposal import B200Proposer, PlainProposer
    g, p = _fixture_patch()
    p.return_residual = True
    p.send_to_device()
    for k in (0, 1):
        prop = g["proposal_%d" % k]
        chi2, dchi2, res = B200Proposer().evaluate_proposal(prop, patch=p, unpack=False)
        sc = band_scales(p, g["f64_residual_%d" % k])
        assert chi2_raw_err(chi2, g["f64_chi2_%d" % k], sc) < CHI2_F64
        assert grad_err(dchi2, g["f64_dchi2_%d" % k]) < GRAD_F64
        assert ref_gap_explained(chi2, g["ref_chi2_%d" % k], g["f64_chi2_%d" % k], CHI2_F64, sc)
        assert grad_err(dchi2, g["ref_dchi2_%d" % k]) < 1e-4
        peak = np.abs(p.data.astype(np.float64) - g["f64_residual_%d" % k]).max()
        assert np.max(np.abs(res - g["f64_residual_%d" % k])) <= 1e-5 * peak
        c2, d2 = PlainProposer().evaluate_proposal(prop, patch=p)[:2]
        assert grad_err(d2, g["f64_dchi2_%d" % k]) < 1e-4


def test_swap_on_the_reference_image_patch():
    """tests/cswap_test.py:60-100 on the GPU path: after the swap the device
    data is the first residual, and evaluating the same scene again leaves
    data - 2 model."""
    from forcepho_b200.proposal import B200Proposer
    g, p = _fixture_patch()
    p.return_residual = True
    p.send_to_device()
    prop = g["proposal_0"]
    pr = B200Proposer()
    _, _, res0 = pr.evaluate_proposal(prop, patch=p, unpack=False)
    data0 = p.data.copy()
    p.swap_on_device()
    assert np.allclose(p.retrieve_array("data"), res0)
    assert np.allclose(p.retrieve_array("residual"), data0)
    _, _, res1 = pr.evaluate_proposal(prop, patch=p, unpack=False)
    model = data0 - res0
    assert np.allclose(res1, data0 - 2 * model, rtol=0, atol=1e-5 * np.abs(model).max())


def test_packed_fits_set_in_a_batch_with_synthetic_patches(tmp_path):
    from test_stores import _PSF, make_image_set
    from forcepho_b200 import synthetic as S
    from forcepho_b200.batch import BatchedProposer
    from forcepho_b200.stores.patch import FITSPatch
    from forcepho_b200.stores.region import CircularRegion
    paths = make_image_set(tmp_path, seed=8)
    p = FITSPatch(fitsfiles=paths)
    p.psfstore = _PSF()
    cat = np.zeros(2, dtype=[(c, np.float64) for c in ("ra", "dec", "q", "pa", "sersic", "rhalf", "B0", "B1")])
    cat["ra"], cat["dec"] = [53.1, 53.1 + 4e-5], [-27.8, -27.8 + 2e-5]
    cat["q"], cat["pa"], cat["sersic"], cat["rhalf"] = [0.8, 0.5], [0.2, 1.0], [2.5, 1.2], [0.12, 0.2]
    cat["B0"], cat["B1"] = [20.0, 8.0], [15.0, 6.0]
    p.build_patch(CircularRegion(53.1, -27.8, 0.6 / 3600.0), cat, allbands=["B0", "B1"])
    # data = the catalog's model (FP64 oracle) + the image noise already packed
    p.data = (p.data + O.render(p, p.scene.get_proposal())).astype(np.float32)
    q = S.config_multiband(seed=12, n_sources=3, n_bands=2, exp_per_band=1, size=40)
    patches = [p, q]
    for x in patches:
        x.return_residual = False
        x.send_to_device()
    props = []
    for x in patches:
        pr = x.scene.get_proposal().copy()
        pr["q"] = np.clip(pr["q"] * 0.95, 0.2, 0.99)
        props.append(pr)
    res = BatchedProposer(patches, tile_pixels=256).evaluate_proposals(props)
    for x, prop, (chi2, dchi2) in zip(patches, props, res):
        c64, g64, r64 = O.evaluate(x, prop, precision="f64", return_residual=True)
        assert chi2_raw_err(chi2, c64, band_scales(x, r64)) < CHI2_F64
        assert grad_err(dchi2, g64) < GRAD_F64


def test_render_and_flux_solve_on_a_packed_fits_patch(tmp_path):
    """Store-backed patches take catalogs in absolute coordinates: the GPU
    render and the design matrix of one must match the FP64 model of the
    packed scene, and a noiseless flux solve must return the catalog fluxes."""
    from test_stores import _PSF, make_image_set
    from forcepho_b200.fitting import optimize_fluxes
    from forcepho_b200.stores.patch import FITSPatch
    from forcepho_b200.stores.region import CircularRegion
    paths = make_image_set(tmp_path, seed=8)
    p = FITSPatch(fitsfiles=paths)
    p.psfstore = _PSF()
    cat = np.zeros(2, dtype=[(c, np.float64) for c in ("ra", "dec", "q", "pa", "sersic", "rhalf", "B0", "B1")])
    cat["ra"], cat["dec"] = [53.1, 53.1 + 4e-5], [-27.8, -27.8 + 2e-5]
    cat["q"], cat["pa"], cat["sersic"], cat["rhalf"] = [0.8, 0.5], [0.2, 1.0], [2.5, 1.2], [0.12, 0.2]
    cat["B0"], cat["B1"] = [20.0, 8.0], [15.0, 6.0]
    p.build_patch(CircularRegion(53.1, -27.8, 0.6 / 3600.0), cat, allbands=["B0", "B1"])
    want = O.render(p, p.scene.get_proposal())
    p.return_residual = True
    p.send_to_device()
    got = np.concatenate(p.render(cat))
    assert np.max(np.abs(got - want)) <= 1e-5 * np.max(np.abs(want))
    live = p.ierr > 0
    p.data = np.where(live, want, 0.0).astype(np.float32)
    p.send_to_device()
    fluxes, precisions = optimize_fluxes(p, cat)
    for b, name in enumerate(p.bandlist):
        np.testing.assert_allclose(fluxes[b], cat[name], rtol=1e-4)
