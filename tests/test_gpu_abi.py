"""fp_evaluate_proposal, the entry point with the kernel ABI of the reference's
EvaluateProposal (forcepho/src/compute_gaussians_kernel.cu:212-214), through
the C ABI: the results of fp_evaluate_proposal_plain (up to the order of
that kernel's shared-memory atomics, as in the reference's kernel), and a
clear error when n_sources disagrees with the patch."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_kernel_abi_entry_point_matches_plain():
    import torch
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    from forcepho_b200.kernel_limits import MAXSOURCES, NPARAMS
    from oracle import oracle as O
    L = N.load()
    p = S.config_multiband(seed=70, render=lambda pp, pr: O.render(pp, pr, precision="f64"), n_sources=5,
                           n_bands=3, exp_per_band=2, size=40)
    p.return_residual = False
    p.send_to_device()
    prop = p.scene.get_proposal().copy()
    prop["q"] *= 0.95
    d_prop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    nb, ns = p.n_bands, int(p.n_sources)
    out = []
    for name in ("fp_evaluate_proposal", "fp_evaluate_proposal_plain"):
        chi2 = torch.zeros(nb, dtype=torch.float64, device="cuda")
        resp = torch.zeros((nb, MAXSOURCES * NPARAMS), dtype=torch.float32, device="cuda")
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        if name == "fp_evaluate_proposal":
            rc = L.fp_evaluate_proposal(p.device_patch_ptr, d_prop.data_ptr(), ns, nb, chi2.data_ptr(),
                                        resp.data_ptr(), s)
        else:
            rc = L.fp_evaluate_proposal_plain(p.device_patch_ptr, d_prop.data_ptr(), nb,
                                              p.max_gauss_per_exposure(), chi2.data_ptr(), resp.data_ptr(), s)
        assert rc == 0, L.fp_error_string()
        torch.cuda.synchronize()
        out.append((chi2.cpu().numpy(), resp.cpu().numpy()))
    np.testing.assert_allclose(out[0][0], out[1][0], rtol=1e-12, atol=0)
    g0, g1 = out[0][1][:, :ns * NPARAMS], out[1][1][:, :ns * NPARAMS]
    assert np.max(np.abs(g0 - g1)) <= 1e-5 * np.max(np.abs(g1))
    c64, g64, _ = O.evaluate(p, prop, precision="f64")
    assert np.all(np.isfinite(out[0][0])) and np.max(np.abs(out[0][0] - c64)) / np.max(np.abs(c64)) < 1e-4
    # n_sources that disagrees with the patch struct: an argument error, nothing launched
    chi2 = torch.zeros(nb, dtype=torch.float64, device="cuda")
    resp = torch.zeros((nb, MAXSOURCES * NPARAMS), dtype=torch.float32, device="cuda")
    rc = L.fp_evaluate_proposal(p.device_patch_ptr, d_prop.data_ptr(), ns + 1, nb, chi2.data_ptr(),
                                resp.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == N.FP_ERR_ARGUMENT
    assert b"n_sources" in L.fp_error_string()
