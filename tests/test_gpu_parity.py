"""Parity of the CUDA kernels (through the C ABI) with the oracle and with the
reference CPU kernel's golden outputs, plus the reference's own known-answer
checks (tests/verification/verify_reference.py:172-184, tests/cswap_test.py:43-110)
restated on the GPU path."""

import numpy as np
import pytest

from conftest import patch_from_golden
from oracle import oracle as O
from tolerances import (CHI2_F64, CHI2_REF, GRAD_F64, GRAD_REF, band_scales, chi2_err, chi2_raw_err, chi2_scale,
                        grad_err, ref_gap_explained)

pytestmark = pytest.mark.gpu


def device_patch(p, return_residual=True):
    p.return_residual = return_residual
    p.send_to_device()
    return p


def proposers():
    from forcepho_b200.proposal import B200Proposer, PlainProposer
    return {"tiled": B200Proposer(), "plain": PlainProposer()}


def check_against(name, chi2, dchi2, res, p, ref_chi2, ref_dchi2, f64_chi2, f64_dchi2):
    scale = chi2_scale(chi2, p.data, p.ierr, res)
    e_ref_c, e_ref_g = chi2_err(chi2, ref_chi2, scale), grad_err(dchi2, ref_dchi2)
    e64_g = grad_err(dchi2, f64_dchi2)
    sc = band_scales(p, res)
    raw64 = chi2_raw_err(chi2, f64_chi2, sc)
    assert e_ref_c < CHI2_REF, (name, "chi2 vs reference", e_ref_c)
    assert e_ref_g < GRAD_REF, (name, "grad vs reference", e_ref_g)
    tol_c, tol_g = (CHI2_F64, GRAD_F64) if name == "tiled" else (CHI2_REF, GRAD_REF)
    assert raw64 < tol_c, (name, "raw chi2 vs f64", raw64)
    assert e64_g < tol_g, (name, "grad vs f64", e64_g)
    assert ref_gap_explained(chi2, ref_chi2, f64_chi2, tol_c, sc), (name, chi2, ref_chi2, f64_chi2)
    return e_ref_c, e_ref_g, raw64, e64_g


@pytest.mark.parametrize("fixture", ["golden_small", "golden_reduced"])
@pytest.mark.parametrize("kind", ["tiled", "plain"])
def test_golden_parity(fixture, kind, request):
    g = request.getfixturevalue(fixture)
    p = device_patch(patch_from_golden(g))
    prop = proposers()[kind]
    for k in (0, 1):
        chi2, dchi2, res = prop.evaluate_proposal(g[f"proposal_{k}"], patch=p, unpack=False)
        assert chi2.dtype == np.float64 and dchi2.dtype == np.float32
        assert dchi2.shape == (p.n_bands, int(p.n_sources), 7)
        check_against(kind, chi2, dchi2, res, p, g[f"ref_chi2_{k}"], g[f"ref_dchi2_{k}"],
                      g[f"f64_chi2_{k}"], g[f"f64_dchi2_{k}"])
        # residuals: against the FP64 oracle's
        model_peak = np.abs(g["data"].astype(np.float64) - g[f"f64_residual_{k}"]).max()
        np.testing.assert_allclose(res, g[f"f64_residual_{k}"], rtol=0, atol=1e-5 * model_peak + 1e-6)


@pytest.mark.parametrize("kind", ["tiled", "plain"])
def test_multiband_full_parity(kind, golden_multiband):
    p, g = golden_multiband
    p = device_patch(p)
    prop = proposers()[kind]
    for k in (0, 1):
        chi2, dchi2, res = prop.evaluate_proposal(g[f"proposal_{k}"], patch=p, unpack=False)
        check_against(kind, chi2, dchi2, res, p, g[f"ref_chi2_{k}"], g[f"ref_dchi2_{k}"],
                      g[f"f64_chi2_{k}"], g[f"f64_dchi2_{k}"])


def test_repeatable_and_deterministic(golden_reduced):
    """Same inputs twice give bitwise-equal results (fixed-order reductions)."""
    p = device_patch(patch_from_golden(golden_reduced))
    prop = proposers()["tiled"]
    a = prop.evaluate_proposal(golden_reduced["proposal_1"], patch=p, unpack=False)
    b = prop.evaluate_proposal(golden_reduced["proposal_1"], patch=p, unpack=False)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_chi2_convention(golden_reduced):
    """Returned chi2 = sum (r^2 - d^2) ierr^2 over each band's pixels, with r the
    returned residual (verify_reference.py:178-184)."""
    g = golden_reduced
    p = device_patch(patch_from_golden(g))
    chi2, _, res = proposers()["tiled"].evaluate_proposal(g["proposal_1"], patch=p, unpack=False)
    for b in range(p.n_bands):
        e0, ne = int(p.band_start[b]), int(p.band_N[b])
        s0 = int(p.exposure_start[e0])
        s1 = int(p.exposure_start[e0 + ne - 1] + p.exposure_N[e0 + ne - 1])
        r = res[s0:s1].astype(np.float64) * p.ierr[s0:s1]
        d = p.data[s0:s1].astype(np.float64) * p.ierr[s0:s1]
        direct = np.sum((r - d) * (r + d))
        scale = np.sum(r * r + d * d)
        assert abs(chi2[b] - direct) <= 3e-7 * scale


def test_swap_semantics(golden_reduced):
    """tests/cswap_test.py:43-110 on the device path: after swap_on_device the
    device data is the previous residual, and a second evaluation gives
    data - 2 model."""
    g = golden_reduced
    p = device_patch(patch_from_golden(g))
    prop = proposers()["tiled"]
    prop0 = g["proposal_0"]
    _, _, residual_original = prop.evaluate_proposal(prop0, patch=p, unpack=False)
    data_original = p.data.copy()
    p.swap_on_device()
    data_postswap = p.retrieve_array("data")
    residual_postswap = p.retrieve_array("residual")
    assert np.array_equal(residual_original, data_postswap)
    assert np.array_equal(data_original, residual_postswap)
    _, _, residual_new = prop.evaluate_proposal(prop0, patch=p, unpack=False)
    model = data_original.astype(np.float64) - residual_original
    np.testing.assert_allclose(residual_new, data_original - 2 * model, rtol=0,
                               atol=1e-5 * np.abs(model).max() + 1e-6)


def test_graph_replay_equals_eager(golden_reduced):
    """The proposer's CUDA-graph replay (upload, three launches, read-back) and
    the same calls issued one by one give identical results, across changing
    proposals and across a data/residual swap (the struct is rewritten in
    place, so the captured graph stays valid)."""
    from forcepho_b200.proposal import B200Proposer
    g = golden_reduced
    pa, pb = device_patch(patch_from_golden(g)), device_patch(patch_from_golden(g))
    eager, graph = B200Proposer(use_graph=False), B200Proposer()
    for swap in (False, True):
        if swap:
            pa.swap_on_device()
            pb.swap_on_device()
        for key in ("proposal_0", "proposal_1", "proposal_0"):
            ca, ga, ra = eager.evaluate_proposal(g[key], patch=pa, unpack=False)
            cb, gb, rb = graph.evaluate_proposal(g[key], patch=pb, unpack=False)
            np.testing.assert_array_equal(ca, cb)
            np.testing.assert_array_equal(ga, gb)
            np.testing.assert_array_equal(ra, rb)
    assert graph._graph is not None and eager._graph is None


def test_culling_and_tile_sizes_agree(golden_multiband):
    """Culling only drops pairs past the cutoff, and the tile size only changes
    summation order: all variants agree far inside the f64 tolerance."""
    from forcepho_b200 import _native as N
    from forcepho_b200.proposal import B200Proposer
    p, g = golden_multiband
    p = device_patch(p, return_residual=False)
    base = None
    for tp in (256, 512, 1024):
        for flags in (0, N.FLAG_NO_CULL, N.FLAG_STATIC):
            chi2, dchi2 = B200Proposer(tile_pixels=tp, flags=flags).evaluate_proposal(g["proposal_1"], patch=p)
            if base is None:
                base = (chi2, dchi2)
                continue
            # different summation groupings: within FP32 rounding of the residuals
            scale = float(np.sum((p.data.astype(np.float64) * p.ierr) ** 2))
            assert np.max(np.abs(chi2 - base[0])) / scale < 1e-7, (tp, flags)
            assert grad_err(dchi2, base[1]) < 1e-6, (tp, flags)


def test_residual_and_unpack(golden_reduced):
    g = golden_reduced
    p = device_patch(patch_from_golden(g))
    chi2, dchi2, res = proposers()["tiled"].evaluate_proposal(g["proposal_0"], patch=p, unpack=True)
    assert isinstance(res, list) and len(res) == p.n_exp
    assert [len(r) for r in res] == list(p.exposure_N)
    p.return_residual = False
    out = proposers()["tiled"].evaluate_proposal(g["proposal_0"], patch=p)
    assert len(out) == 2


def test_status_word_clean(golden_reduced):
    from forcepho_b200.proposal import B200Proposer
    p = device_patch(patch_from_golden(golden_reduced))
    prop = B200Proposer()
    prop.evaluate_proposal(golden_reduced["proposal_0"], patch=p)
    assert prop._plan.read_status() == 0


def test_unpadded_and_empty_exposures():
    """Exposures not padded to 32 (scalar pixel loads), an empty exposure, a
    source far outside the image (every Gaussian culled) -- edge cases the
    reference only meets with its own padding."""
    from forcepho_b200 import synthetic as S
    rng = np.random.default_rng(11)
    p = S.make_patch(rng, n_sources=3, exp_per_band=[2, 1], exp_pix=[(37, 29), (41, 23), (19, 13)],
                     n_psf=2, source_params=S._broad_source)
    # drop the 32-padding of exposure 0 and empty exposure 2
    keep = np.ones(p.npix, bool)
    n0 = 37 * 29
    keep[n0:int(p.exposure_N[0])] = False
    for n in ["xpix", "ypix"]:
        setattr(p, n, getattr(p, n)[keep])
    p.exposure_N = np.array([n0, p.exposure_N[1], 0], np.int32)
    p.exposure_start = np.array([0, n0, n0 + p.exposure_N[1]], np.int32)
    p.xpix, p.ypix = p.xpix[:p.exposure_start[2]], p.ypix[:p.exposure_start[2]]
    p.data = np.zeros(len(p.xpix), np.float32)
    p.ierr = np.ones(len(p.xpix), np.float32)
    p.original_shapes = [(37, 29, n0), (41, 23, int(p.exposure_N[1])), (19, 13, 0)]
    S.add_noise(p, rng, 1.0, O.render(p, p.scene.get_proposal()))
    prop = p.scene.get_proposal().copy()
    prop["ra"][2] += 0.05                               # ~6000 px away
    ref = O.ref_evaluate(p, prop, return_residual=True)
    f64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    p = device_patch(p)
    for kind, pr in proposers().items():
        chi2, dchi2, res = pr.evaluate_proposal(prop, patch=p, unpack=False)
        check_against(kind, chi2, dchi2, res, p, ref[0], ref[1], f64[0], f64[1])
        assert np.all(dchi2[:, 2] == 0)
