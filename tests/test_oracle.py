"""The oracle pinned against the reference's own outputs (CPU only).

The golden fixtures hold outputs of the reference CPU kernel
(forcepho/src/compute_gaussians_kernel.cc, compiled from source) on seeded
synthetic patches; see tests/golden/make_golden.py.
"""

import numpy as np
import pytest

from conftest import patch_from_golden
from oracle import oracle as O
from tolerances import chi2_err, chi2_scale, grad_err


@pytest.mark.parametrize("fixture", ["golden_small", "golden_reduced"])
@pytest.mark.parametrize("k", [0, 1])
def test_oracle_f32_matches_reference_kernel(fixture, k, request):
    g = request.getfixturevalue(fixture)
    p = patch_from_golden(g)
    prop = g[f"proposal_{k}"]
    chi2, dchi2, res = O.evaluate(p, prop, precision="f32", return_residual=True, nthreads=1)
    scale = chi2_scale(chi2, p.data, np.tile(p.ierr, 1), res)
    # same arithmetic as the reference, only libm/compiler differences remain
    assert chi2_err(chi2, g[f"ref_chi2_{k}"], scale) < 1e-9
    assert grad_err(dchi2, g[f"ref_dchi2_{k}"]) < 1e-6
    np.testing.assert_allclose(res, g[f"ref_residual_{k}"], rtol=0, atol=1e-6 * np.abs(p.data).max())


@pytest.mark.parametrize("fixture", ["golden_small", "golden_reduced"])
def test_oracle_f64_reproducible(fixture, request):
    g = request.getfixturevalue(fixture)
    p = patch_from_golden(g)
    for k in (0, 1):
        chi2, dchi2, res = O.evaluate(p, g[f"proposal_{k}"], precision="f64", return_residual=True)
        np.testing.assert_allclose(chi2, g[f"f64_chi2_{k}"], rtol=1e-12, atol=0)
        np.testing.assert_allclose(dchi2, g[f"f64_dchi2_{k}"], rtol=1e-10, atol=1e-12 * np.abs(dchi2).max())


@pytest.mark.parametrize("fixture", ["golden_small", "golden_reduced"])
def test_reference_kernel_vs_f64(fixture, request):
    """The reference FP32 kernel itself sits within the parity tolerances of the
    FP64 oracle (so those tolerances are attainable)."""
    g = request.getfixturevalue(fixture)
    p = patch_from_golden(g)
    for k in (0, 1):
        scale = chi2_scale(g[f"f64_chi2_{k}"], p.data, p.ierr, g[f"f64_residual_{k}"])
        assert chi2_err(g[f"ref_chi2_{k}"], g[f"f64_chi2_{k}"], scale) < 1e-5
        assert grad_err(g[f"ref_dchi2_{k}"], g[f"f64_dchi2_{k}"]) < 1e-4


def test_slow_path_model_matches(golden_small):
    """forcepho/slow/gaussmodel.py's per-Gaussian pixel evaluation (FP64, no
    cutoff) agrees with the FP64 oracle's model away from the cutoff."""
    g = golden_small
    model_f64 = g["data"].astype(np.float64) - g["f64_residual_0"].astype(np.float64)
    n = int(g["exposure_N"][0])
    slow = g["slow_model_0"][:n]
    peak = np.abs(slow).max()
    np.testing.assert_allclose(model_f64[:n], slow, rtol=0, atol=2e-6 * peak)


def test_multiband_fixture_inputs(golden_multiband):
    p, g = golden_multiband
    assert p.n_bands == 5 and p.n_exp == 10 and int(p.n_sources) == 16
    assert p.n_pairs() == 225280 * 576


@pytest.mark.slow
def test_oracle_multiband_full(golden_multiband):
    p, g = golden_multiband
    chi2, dchi2, res = O.evaluate(p, g["proposal_1"], precision="f32", return_residual=True)
    scale = chi2_scale(chi2, p.data, p.ierr, res)
    assert chi2_err(chi2, g["ref_chi2_1"], scale) < 1e-8
    assert grad_err(dchi2, g["ref_dchi2_1"]) < 1e-5


def test_count_pairs_small(golden_small):
    p = patch_from_golden(golden_small)
    tot, act = O.count_pairs(p, golden_small["proposal_0"])
    assert tot == 4096 * 27
    assert 0 < act < tot
