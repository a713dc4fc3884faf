"""fp_evaluate_batch_noalloc: the evaluation for callers that cannot allocate
device memory (for example a binding that only holds raw pointers from another
runtime, or a process whose device memory belongs to another allocator's pool).
It uses a fixed device array instead of a caller workspace.  Checked through
the C ABI against fp_evaluate_batch, on two calls in a row with different
proposals (the array keeps the previous call's contents), plus the size limit.
This file is collected last on purpose."""

import ctypes

import numpy as np
import pytest

from tolerances import CHI2_F64, GRAD_F64, grad_err

pytestmark = pytest.mark.gpu


def _perturbed(prop, seed):
    rng = np.random.default_rng(seed)
    q = prop.copy()
    q["q"] = np.clip(q["q"] * rng.uniform(0.9, 1.1, len(q)), 0.2, 0.99).astype(np.float32)
    q["fluxes"] *= rng.uniform(0.8, 1.2, q["fluxes"].shape).astype(np.float32)
    return q


def test_noalloc_matches_workspace_entry_point():
    import torch
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    from forcepho_b200.device import Plan, pack_proposals

    L = N.load()
    p = S.config_multiband(seed=2)
    p.return_residual = False
    p.send_to_device()
    plan = Plan([p], tile_pixels=1024)
    assert plan.sizes.workspace_bytes <= N.NOALLOC_WORKSPACE_BYTES
    launch = plan.launch(ctas_per_sm=3)
    stream = torch.cuda.current_stream()
    scale = float(np.sum((p.data.astype(np.float64) * p.ierr) ** 2))
    prop0 = p.scene.get_proposal()

    for call, seed in enumerate((1, 2)):        # two calls in a row, different proposals
        host = pack_proposals([_perturbed(prop0, seed)], 1)
        plan.proposals.copy_(torch.from_numpy(host.view(np.uint8).reshape(-1)))
        plan.evaluate(launch, stream=stream)           # the existing entry point
        chi2_ref = plan.chi2.clone()
        resp_ref = plan.response.clone()
        chi2 = torch.full_like(plan.chi2, np.nan)
        resp = torch.full_like(plan.response, np.nan)
        rc = L.fp_evaluate_batch_noalloc(plan.d_patches.data_ptr(), 1, ctypes.byref(plan.sizes),
                                         ctypes.byref(plan.tables), plan.proposals.data_ptr(), chi2.data_ptr(),
                                         resp.data_ptr(), ctypes.byref(launch), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.fp_error_string().decode()
        torch.cuda.synchronize()
        nb, ns = p.n_bands, int(p.n_sources)
        c, cr = chi2.cpu().numpy()[0, :nb], chi2_ref.cpu().numpy()[0, :nb]
        g = resp.cpu().numpy()[0].reshape(30, 30, 7)[:nb, :ns]
        gr = resp_ref.cpu().numpy()[0].reshape(30, 30, 7)[:nb, :ns]
        assert np.all(np.isfinite(c)) and np.all(np.isfinite(g)), call
        assert np.max(np.abs(c - cr)) / scale < CHI2_F64, call
        assert grad_err(g, gr) < GRAD_F64, call


def test_noalloc_rejects_plans_beyond_the_array():
    from forcepho_b200 import _native as N
    L = N.load()
    sz = N.PlanSizes(1, 1, 1, 1, 1, 1, 1, N.NOALLOC_WORKSPACE_BYTES + 256, 1)
    lp = N.Launch(1024, 3, 0, 0)
    rc = L.fp_evaluate_batch_noalloc(None, 1, ctypes.byref(sz), None, None, None, None, ctypes.byref(lp), None)
    assert rc == N.FP_ERR_WORKSPACE
    assert "fixed" in L.fp_error_string().decode()
