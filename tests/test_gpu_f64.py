"""The FP64 device evaluation (fp_evaluate_proposal_f64) against the FP64
oracle: the same model in the same precision, so chi2 and gradients agree to
the summation-order level (1e-11 of chi2, 1e-9 of the gradient), on the golden
fixtures, on the full multiband workload and at detector-scale coordinates.
It then serves as the reference for the tiled FP32 kernels on patches too large
for the oracle."""

import ctypes

import numpy as np
import pytest

from conftest import patch_from_golden
from oracle import oracle as O
from tolerances import CHI2_F64, GRAD_F64, band_scales, chi2_raw_err, grad_err

pytestmark = pytest.mark.gpu

CHI2_EXACT = 1e-11
GRAD_EXACT = 1e-9


def _device(p, return_residual=False):
    p.return_residual = return_residual
    p.send_to_device()
    return p


@pytest.mark.parametrize("fixture", ["golden_small", "golden_reduced"])
def test_golden_fixtures_in_fp64(fixture, request):
    from forcepho_b200.proposal import F64Proposer
    g = request.getfixturevalue(fixture)
    p = _device(patch_from_golden(g))
    f64 = F64Proposer()
    for k in (0, 1):
        chi2, dchi2 = f64.evaluate_proposal(g[f"proposal_{k}"], patch=p)
        assert chi2.dtype == np.float64 and dchi2.dtype == np.float64
        assert dchi2.shape == (p.n_bands, int(p.n_sources), 7)
        sc = band_scales(p, g[f"f64_residual_{k}"])
        assert chi2_raw_err(chi2, g[f"f64_chi2_{k}"], sc) < CHI2_EXACT
        assert grad_err(dchi2, g[f"f64_dchi2_{k}"]) < GRAD_EXACT


def test_multiband_workload_in_fp64(golden_multiband):
    from forcepho_b200.proposal import F64Proposer
    p, g = golden_multiband
    p = _device(p)
    for k in (0, 1):
        chi2, dchi2 = F64Proposer(p).evaluate_proposal(g[f"proposal_{k}"])
        # sum (r^2 + d^2) ierr^2 = chi2 + 2 sum d^2 ierr^2 (the fixture keeps no residual)
        sc = g[f"f64_chi2_{k}"] + 2.0 * band_scales(p, np.zeros(p.npix))
        assert chi2_raw_err(chi2, g[f"f64_chi2_{k}"], sc) < CHI2_EXACT
        assert grad_err(dchi2, g[f"f64_dchi2_{k}"]) < GRAD_EXACT


@pytest.mark.parametrize("offset", [(0.0, 0.0), (7000.0, 6000.0)])
def test_fp64_far_from_the_origin(offset):
    from forcepho_b200.proposal import F64Proposer
    from test_gpu_coordinates import _patch
    p, prop = _patch(5, offset)
    p = _device(p)
    chi2, dchi2 = F64Proposer().evaluate_proposal(prop, patch=p)
    c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    assert chi2_raw_err(chi2, c64, band_scales(p, r64)) < CHI2_EXACT
    assert grad_err(dchi2, g64) < GRAD_EXACT


def test_tiled_kernels_against_fp64_on_large_patches():
    """The FP32 tiled path against the device FP64 evaluation on the bench's
    patch shape (too slow for the CPU oracle at this count), with the FP64
    tolerances the tiled path meets against the oracle."""
    from forcepho_b200 import synthetic as S
    from forcepho_b200.proposal import B200Proposer, F64Proposer
    tiled, f64 = B200Proposer(), F64Proposer()
    for seed in (11, 12, 13):
        p = S.config_multiband(seed=seed)
        p = _device(p, return_residual=True)
        prop = p.scene.get_proposal()
        prop["q"] = np.clip(prop["q"] * 0.97, 0.2, 0.99)
        prop["ra"] += 3e-6
        c32, g32, res = tiled.evaluate_proposal(prop, patch=p, unpack=False)
        c64, g64 = f64.evaluate_proposal(prop, patch=p)
        assert chi2_raw_err(c32, c64, band_scales(p, res)) < CHI2_F64
        assert grad_err(g32, g64) < GRAD_F64


def test_gaussian_count_over_the_plan_sets_the_status():
    """Exposures with more image Gaussians than the caller's maximum (here
    every exposure: all bands have 4 PSF components) are skipped and flagged,
    with the outputs left cleared."""
    import torch
    from forcepho_b200 import _native as N
    from forcepho_b200.device import current_stream_ptr
    from forcepho_b200.kernel_limits import MAXBANDS, MAXSOURCES, NPARAMS
    from forcepho_b200.structs import source_struct_dtype
    from test_gpu_coordinates import _patch
    p, prop = _patch(6, (0.0, 0.0))
    p = _device(p)
    L = N.load()
    max_gauss = p.max_gauss_per_exposure() - 1
    n = ctypes.c_size_t()
    N.check(L.fp_f64_workspace_bytes(p.n_exp, max_gauss, ctypes.byref(n)), "workspace")
    ws = torch.zeros(n.value, dtype=torch.uint8, device="cuda")
    host = np.zeros(len(prop), dtype=source_struct_dtype)
    host[:] = prop
    d_prop = torch.from_numpy(host.view(np.uint8).copy()).cuda()
    chi2 = torch.full((MAXBANDS,), 7.0, dtype=torch.float64, device="cuda")
    dchi2 = torch.full((MAXBANDS, MAXSOURCES * NPARAMS), 7.0, dtype=torch.float64, device="cuda")
    s = current_stream_ptr(None)
    N.check(L.fp_evaluate_proposal_f64(ctypes.c_void_p(p.device_patch_ptr), ctypes.c_void_p(d_prop.data_ptr()),
                                       p.n_bands, p.n_exp, max_gauss, ctypes.c_void_p(chi2.data_ptr()),
                                       ctypes.c_void_p(dchi2.data_ptr()), ctypes.c_void_p(ws.data_ptr()), n.value, s),
            "fp_evaluate_proposal_f64")
    st = ctypes.c_int32()
    N.check(L.fp_read_status(ctypes.c_void_p(ws.data_ptr()), ctypes.byref(st), s), "fp_read_status")
    assert st.value == N.STATUS_GAUSS_COUNT
    # outputs were cleared and nothing was added for the rejected exposures
    assert torch.all(chi2[:p.n_bands] == 0) and torch.all(dchi2[:p.n_bands] == 0)
    # the status word was cleared by the read; a sized call evaluates every band
    from forcepho_b200.proposal import F64Proposer
    c, _ = F64Proposer().evaluate_proposal(prop, patch=p)
    assert np.all(c != 0)


@pytest.mark.timeout(900)
def test_whole_batched_workload_against_fp64():
    """Full-size parity: all 512 patches of the batched workload (1.04e11
    pixel-Gaussian pairs), evaluated by the batched FP32 path in one launch
    set, against the device FP64 evaluation patch by patch, with the FP64
    tolerances of the parity tests.  Raw chi2 per band is measured against
    max(|chi2|, RAW_FLOOR sum (r^2 + d^2) ierr^2), where sum (r^2 + d^2) ierr^2
    = chi2_f64 + 2 sum d^2 ierr^2."""
    from forcepho_b200 import synthetic as S
    from forcepho_b200.batch import BatchedProposer, render_models
    from forcepho_b200.proposal import F64Proposer
    patches = []
    for sh in S.batched_shapes(seed=4, n_patches=512):
        rng = np.random.default_rng(sh["seed"])
        p = S.make_patch(rng, n_sources=sh["n_sources"], exp_per_band=sh["exp_per_band"], exp_pix=sh["exp_pix"],
                         n_psf=4, source_params=S._broad_source, raster_width=256)
        p._rng = rng
        patches.append(p)
    sigmas = [p._rng.uniform(0.5, 2.0, p.n_exp) for p in patches]
    for p, m, sg in zip(patches, render_models(patches), sigmas):
        S.add_noise(p, p._rng, sg, m)
        _device(p)
    rng = np.random.default_rng(99)
    proposals = []
    for p in patches:
        q = p.scene.get_proposal().copy()
        q["ra"] += rng.normal(0, 2e-6, len(q)).astype(np.float32)
        q["dec"] += rng.normal(0, 2e-6, len(q)).astype(np.float32)
        q["q"] = np.clip(q["q"] * rng.uniform(0.95, 1.05, len(q)), 0.2, 0.99).astype(np.float32)
        proposals.append(q)
    got = BatchedProposer(patches, tile_pixels=1024, autotune=False).evaluate_proposals(proposals)
    f64 = F64Proposer()
    worst_c, worst_g = 0.0, 0.0
    for i, (p, q) in enumerate(zip(patches, proposals)):
        c64, g64 = f64.evaluate_proposal(q, patch=p)
        c32, g32 = got[i]
        sc = c64 + 2.0 * band_scales(p, np.zeros(p.npix))
        worst_c = max(worst_c, chi2_raw_err(c32, c64, sc))
        worst_g = max(worst_g, grad_err(g32, g64))
        p.free()
    assert worst_c < CHI2_F64, worst_c
    assert worst_g < GRAD_F64, worst_g
