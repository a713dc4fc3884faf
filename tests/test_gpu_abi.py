"""fp_evaluate_proposal, the entry point with the kernel ABI of the reference's
EvaluateProposal (forcepho/src/compute_gaussians_kernel.cu:212-214), through
the C ABI.  It runs the tiled kernels on a plan the library keeps per patch:
checked against the FP64 oracle on the small, multiband and limits-size
patches, bitwise against B200Proposer (same plan rule, same kernels), across a
data/residual swap and a re-upload (the cached plan must follow the patch), and
for a clear error when n_sources disagrees with the patch."""

import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import (CHI2_F64, CHI2_REF, GRAD_F64, GRAD_REF, band_scales, chi2_err, chi2_raw_err, chi2_scale,
                        grad_err)

pytestmark = pytest.mark.gpu


def _call(L, p, prop, nb=None):
    import torch
    from forcepho_b200.kernel_limits import MAXSOURCES, NPARAMS
    nb = nb or p.n_bands
    d_prop = torch.from_numpy(np.ascontiguousarray(prop).view(np.uint8).copy()).cuda()
    chi2 = torch.full((nb,), np.nan, dtype=torch.float64, device="cuda")
    resp = torch.full((nb, MAXSOURCES * NPARAMS), np.nan, dtype=torch.float32, device="cuda")
    rc = L.fp_evaluate_proposal(p.device_patch_ptr, d_prop.data_ptr(), int(p.n_sources), nb, chi2.data_ptr(),
                                resp.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.fp_error_string()
    torch.cuda.synchronize()
    ns = int(p.n_sources)
    return chi2.cpu().numpy(), resp.cpu().numpy().reshape(nb, MAXSOURCES, NPARAMS)[:, :ns]


def _check_f64(p, prop, chi2, dchi2, bands=None):
    c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True, bands=bands)
    bands = list(range(p.n_bands)) if bands is None else list(bands)
    sc = band_scales(p, r64)
    assert chi2_raw_err(chi2[bands], c64[bands], sc[bands]) < CHI2_F64
    assert grad_err(dchi2[bands], g64[bands]) < GRAD_F64


def _perturbed(p, f=0.95):
    prop = p.scene.get_proposal().copy()
    prop["q"] = np.clip(prop["q"] * f, 0.2, 0.99)
    return prop


@pytest.mark.parametrize("config", ["small", "multiband"])
def test_kernel_abi_entry_point_is_the_tiled_path(config):
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    from forcepho_b200.proposal import B200Proposer
    L = N.load()
    p = S.CONFIGS[config](seed=3)
    p.return_residual = False
    p.send_to_device()
    prop = _perturbed(p)
    chi2, dchi2 = _call(L, p, prop)
    _check_f64(p, prop, chi2, dchi2)
    # the same plan rule and kernels as the Python proposer: bitwise equal
    c1, g1 = B200Proposer().evaluate_proposal(prop, patch=p)
    assert np.array_equal(chi2, c1) and np.array_equal(dchi2, g1)
    # a second call reuses the cached plan and gives the same bits
    chi2b, dchi2b = _call(L, p, prop)
    assert np.array_equal(chi2, chi2b) and np.array_equal(dchi2, dchi2b)


def test_kernel_abi_entry_point_at_kernel_limits():
    """30 sources, 8 bands x 4 exposures of 256x256 px, 6-Gaussian PSFs; two
    bands checked against the FP64 oracle."""
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    L = N.load()
    p = S.config_limits(seed=4)
    p.return_residual = False
    p.send_to_device()
    prop = _perturbed(p, 0.97)
    chi2, dchi2 = _call(L, p, prop)
    assert chi2.shape == (8,) and dchi2.shape == (8, 30, 7)
    _check_f64(p, prop, chi2, dchi2, bands=(0, 5))


def test_kernel_abi_plan_follows_the_patch():
    """swap_on_device changes the data pointer and re-sends the metadata; a
    re-upload changes every pointer; after each the results match the oracle
    on what the device holds.  Release frees the plans; the next call re-plans
    and gives the same bits."""
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    L = N.load()
    p = S.config_multiband(seed=8, render=lambda pp, pr: O.render(pp, pr, precision="f64"), n_sources=4,
                           n_bands=2, exp_per_band=2, size=48)
    p.return_residual = True
    p.send_to_device()
    prop = _perturbed(p)
    chi2, dchi2 = _call(L, p, prop)
    _check_f64(p, prop, chi2, dchi2)
    # the device data becomes this evaluation's residual
    res = p.retrieve_array("residual")
    p.swap_on_device()
    data_host = p.data
    p.data = res
    chi2s, dchi2s = _call(L, p, prop)
    _check_f64(p, prop, chi2s, dchi2s)
    p.data = data_host
    assert not np.array_equal(chi2s, chi2)
    # a fresh upload (new device arrays) of other pixel values
    p.data = (p.data * 1.5).astype(np.float32)
    p.send_to_device()
    chi2u, dchi2u = _call(L, p, prop)
    _check_f64(p, prop, chi2u, dchi2u)
    assert L.fp_evaluate_proposal_release() == 0
    chi2r, dchi2r = _call(L, p, prop)
    assert np.array_equal(chi2r, chi2u) and np.array_equal(dchi2r, dchi2u)


def test_kernel_abi_rejects_inconsistent_source_count():
    import torch
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    from forcepho_b200.kernel_limits import MAXSOURCES, NPARAMS
    L = N.load()
    p = S.config_small(seed=5)
    p.return_residual = False
    p.send_to_device()
    prop = p.scene.get_proposal()
    d_prop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    nb, ns = p.n_bands, int(p.n_sources)
    chi2 = torch.zeros(nb, dtype=torch.float64, device="cuda")
    resp = torch.zeros((nb, MAXSOURCES * NPARAMS), dtype=torch.float32, device="cuda")
    rc = L.fp_evaluate_proposal(p.device_patch_ptr, d_prop.data_ptr(), ns + 1, nb, chi2.data_ptr(),
                                resp.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == N.FP_ERR_ARGUMENT
    assert b"n_sources" in L.fp_error_string()


def test_plain_comparator_still_matches():
    """fp_evaluate_proposal_plain, the one-CTA-per-band comparator, against the
    tiled reference-ABI call (up to the order of its shared-memory atomics)."""
    import torch
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    from forcepho_b200.kernel_limits import MAXSOURCES, NPARAMS
    L = N.load()
    p = S.config_multiband(seed=70, render=lambda pp, pr: O.render(pp, pr, precision="f64"), n_sources=5,
                           n_bands=3, exp_per_band=2, size=40)
    p.return_residual = False
    p.send_to_device()
    prop = _perturbed(p)
    chi2_t, g_t = _call(L, p, prop)
    d_prop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    nb, ns = p.n_bands, int(p.n_sources)
    chi2 = torch.zeros(nb, dtype=torch.float64, device="cuda")
    resp = torch.zeros((nb, MAXSOURCES * NPARAMS), dtype=torch.float32, device="cuda")
    rc = L.fp_evaluate_proposal_plain(p.device_patch_ptr, d_prop.data_ptr(), nb, p.max_gauss_per_exposure(),
                                      chi2.data_ptr(), resp.data_ptr(),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.fp_error_string()
    torch.cuda.synchronize()
    c_p = chi2.cpu().numpy()
    g_p = resp.cpu().numpy().reshape(nb, MAXSOURCES, NPARAMS)[:, :ns]
    # the comparator computes in FP32 like the reference kernel, whose raw chi2
    # error can pass 1e-5 where chi2 has cancelled; its tolerance is the
    # reference's, relative to sum (r^2 + d^2) ierr^2
    _, _, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    assert chi2_err(c_p, chi2_t, chi2_scale(chi2_t, p.data, p.ierr, r64)) < CHI2_REF
    assert grad_err(g_p, g_t) < GRAD_REF


def test_kernel_abi_plan_cache_evicts_and_replans():
    """More patches than the library keeps plans for (64): the least recently
    used plan is freed, and a later call on its patch re-plans and gives the
    same bits."""
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    L = N.load()
    assert L.fp_evaluate_proposal_release() == 0
    patches = []
    for i in range(66):
        p = S.config_small(seed=100 + i, size=32)
        p.return_residual = False
        p.send_to_device()
        patches.append(p)
    props = [_perturbed(p) for p in patches]
    first = [_call(L, p, q) for p, q in zip(patches, props)]      # 66 plans: the first two evicted
    again = _call(L, patches[0], props[0])
    assert np.array_equal(again[0], first[0][0]) and np.array_equal(again[1], first[0][1])
    _check_f64(patches[0], props[0], *again)
    assert L.fp_evaluate_proposal_release() == 0
