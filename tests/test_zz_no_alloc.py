"""fp_evaluate_batch_noalloc: the evaluation for callers that cannot allocate
device memory (for example a binding that only holds raw pointers from another
runtime, or a process whose device memory belongs to another allocator's pool).
It uses a fixed device array instead of a caller workspace.  Checked through
the C ABI against fp_evaluate_batch, on two calls in a row with different
proposals (the array keeps the previous call's contents), plus the size limit
and the status word of a call whose patch no longer matches its plan.
This file is collected last on purpose."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# byte offset of n_sources in the 152-byte patch struct (after nine pointers)
_N_SOURCES_OFFSET = 72


def _perturbed(prop, seed):
    rng = np.random.default_rng(seed)
    q = prop.copy()
    q["q"] = np.clip(q["q"] * rng.uniform(0.9, 1.1, len(q)), 0.2, 0.99).astype(np.float32)
    q["fluxes"] *= rng.uniform(0.8, 1.2, q["fluxes"].shape).astype(np.float32)
    return q


def _setup():
    import torch
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    from forcepho_b200.device import Plan

    L = N.load()
    p = S.config_multiband(seed=2)
    p.return_residual = False
    p.send_to_device()
    plan = Plan([p], tile_pixels=1024)
    assert plan.sizes.workspace_bytes <= N.NOALLOC_WORKSPACE_BYTES
    return L, N, p, plan, plan.launch(ctas_per_sm=3), torch.cuda.current_stream()


def _noalloc(L, plan, launch, stream, chi2, resp):
    return L.fp_evaluate_batch_noalloc(plan.d_patches.data_ptr(), 1, ctypes.byref(plan.sizes),
                                       ctypes.byref(plan.tables), plan.proposals.data_ptr(), chi2.data_ptr(),
                                       resp.data_ptr(), ctypes.byref(launch), ctypes.c_void_p(stream.cuda_stream))


def _status(L, N, stream):
    st = ctypes.c_int32(-1)
    N.check(L.fp_read_status_noalloc(ctypes.byref(st), ctypes.c_void_p(stream.cuda_stream)),
            "fp_read_status_noalloc")
    return int(st.value)


def _set_proposal(plan, prop):
    import torch
    from forcepho_b200.device import pack_proposals
    host = pack_proposals([prop], 1)
    plan.proposals.copy_(torch.from_numpy(host.view(np.uint8).reshape(-1)))


def test_noalloc_matches_workspace_entry_point():
    """Same tables, same launch parameters, deterministic kernels: the results
    of the two entry points are bitwise equal, call after call."""
    import torch
    L, N, p, plan, launch, stream = _setup()
    prop0 = p.scene.get_proposal()
    nb, ns = p.n_bands, int(p.n_sources)
    for call, seed in enumerate((1, 2)):        # two calls in a row, different proposals
        _set_proposal(plan, _perturbed(prop0, seed))
        plan.evaluate(launch, stream=stream)           # the existing entry point
        chi2_ref = plan.chi2.clone()
        resp_ref = plan.response.clone()
        chi2 = torch.full_like(plan.chi2, np.nan)
        resp = torch.full_like(plan.response, np.nan)
        rc = _noalloc(L, plan, launch, stream, chi2, resp)
        assert rc == 0, L.fp_error_string().decode()
        assert _status(L, N, stream) == 0
        c, cr = chi2.cpu().numpy()[0, :nb], chi2_ref.cpu().numpy()[0, :nb]
        g = resp.cpu().numpy()[0].reshape(30, 30, 7)[:nb, :ns]
        gr = resp_ref.cpu().numpy()[0].reshape(30, 30, 7)[:nb, :ns]
        assert np.all(np.isfinite(c)) and np.all(np.isfinite(g)), call
        assert np.array_equal(c, cr), call
        assert np.array_equal(g, gr), call


def test_noalloc_reports_a_patch_that_no_longer_matches_its_plan():
    """A valid call, then a call whose patch struct claims another source count
    than the plan was made for: the second call reports FP_STATUS_SOURCES and
    returns a zero model (chi2 0, gradient 0), never the first call's values
    left in the shared array.  With the struct restored, results are back."""
    import torch
    L, N, p, plan, launch, stream = _setup()
    nb, ns = p.n_bands, int(p.n_sources)
    _set_proposal(plan, _perturbed(p.scene.get_proposal(), 3))
    chi2_a = torch.full_like(plan.chi2, np.nan)
    resp_a = torch.full_like(plan.response, np.nan)
    assert _noalloc(L, plan, launch, stream, chi2_a, resp_a) == 0, L.fp_error_string().decode()
    assert _status(L, N, stream) == 0
    c_a = chi2_a.cpu().numpy()[0, :nb]
    assert np.all(c_a != 0)

    # the patch struct now disagrees with the plan about n_sources
    struct = p.device_patch
    saved = struct[_N_SOURCES_OFFSET:_N_SOURCES_OFFSET + 4].clone()
    struct[_N_SOURCES_OFFSET:_N_SOURCES_OFFSET + 4].copy_(
        torch.from_numpy(np.array([ns - 1], np.int32).view(np.uint8)))
    try:
        chi2_b = torch.full_like(plan.chi2, np.nan)
        resp_b = torch.full_like(plan.response, np.nan)
        assert _noalloc(L, plan, launch, stream, chi2_b, resp_b) == 0, L.fp_error_string().decode()
        st = _status(L, N, stream)
        assert st & N.STATUS_SOURCES, st
        c_b = chi2_b.cpu().numpy()[0, :nb]
        g_b = resp_b.cpu().numpy()[0].reshape(30, 30, 7)[:nb, :ns]
        assert np.all(c_b == 0.0) and np.all(g_b == 0.0)
        assert _status(L, N, stream) == 0              # reading clears it
    finally:
        struct[_N_SOURCES_OFFSET:_N_SOURCES_OFFSET + 4].copy_(saved)

    chi2_c = torch.full_like(plan.chi2, np.nan)
    resp_c = torch.full_like(plan.response, np.nan)
    assert _noalloc(L, plan, launch, stream, chi2_c, resp_c) == 0, L.fp_error_string().decode()
    assert _status(L, N, stream) == 0
    # rows of bands the patch does not have stay at their NaN fill
    assert np.array_equal(chi2_c.cpu().numpy()[0, :nb], chi2_a.cpu().numpy()[0, :nb])
    assert np.array_equal(resp_c.cpu().numpy()[0, :nb], resp_a.cpu().numpy()[0, :nb])


def test_noalloc_rejects_plans_beyond_the_array():
    from forcepho_b200 import _native as N
    L = N.load()
    sz = N.PlanSizes(1, 1, 1, 1, 1, 1, 1, N.NOALLOC_WORKSPACE_BYTES + 256, 1)
    lp = N.Launch(1024, 3, 0, 0)
    rc = L.fp_evaluate_batch_noalloc(None, 1, ctypes.byref(sz), None, None, None, None, ctypes.byref(lp), None)
    assert rc == N.FP_ERR_WORKSPACE
    assert "fixed" in L.fp_error_string().decode()


def test_noalloc_rejected_call_queues_nothing():
    """Bad arguments are refused before anything is queued on the stream or
    written to the shared array."""
    import torch
    L, N, p, plan, launch, stream = _setup()
    _set_proposal(plan, p.scene.get_proposal())
    chi2 = torch.zeros_like(plan.chi2)
    resp = torch.zeros_like(plan.response)
    assert _noalloc(L, plan, launch, stream, chi2, resp) == 0, L.fp_error_string().decode()
    bad = N.Launch(768, 3, 0, 0)            # not a supported tile size
    rc = L.fp_evaluate_batch_noalloc(plan.d_patches.data_ptr(), 1, ctypes.byref(plan.sizes),
                                     ctypes.byref(plan.tables), plan.proposals.data_ptr(), chi2.data_ptr(),
                                     resp.data_ptr(), ctypes.byref(bad), ctypes.c_void_p(stream.cuda_stream))
    assert rc == N.FP_ERR_ARGUMENT
    assert "tile_pixels" in L.fp_error_string().decode()
    assert _status(L, N, stream) == 0
