"""The differentiable path and device-resident HMC on the GPU.

* ``PatchChi2`` (torch.autograd.Function over the tiled kernels): backward
  equals central finite differences of the FP64 oracle's chi2 and the
  reference CPU kernel's gradient (stack_grad of its Response records).
* ``DeviceHMC``: its device lnp / dlnp/dz equal FastPosterior's on the host
  path (same bounds), graph replay equals eager launches, and short
  trajectories conserve energy to leapfrog accuracy.
"""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# central-difference steps per parameter kind, powers of two so that theta +- h
# is exact in the f32 proposal records (ra/dec: 2^-30 deg ~ 1.1e-4 px)
FD_STEP = {"flux": 2.0 ** -10, "ra": 2.0 ** -30, "dec": 2.0 ** -30, "q": 2.0 ** -14, "pa": 2.0 ** -14,
           "sersic": 2.0 ** -6, "rhalf": 2.0 ** -9}
# sersic and rhalf reach chi2 through the spline amplitudes, rounded to f32 in
# the proposal: one central difference has either truncation (curvature of the
# spline, ~4e-4 at 2^-7) or rounding error (~1e-4 at 2^-12) above 1e-5, so these
# use Richardson extrapolation of steps h and h/2 (error ~1e-5)
RICHARDSON = ("sersic", "rhalf")


def central_difference(f, th, j, h, richardson=False):
    def cd(step):
        tp, tm = th.copy(), th.copy()
        tp[j] += step
        tm[j] -= step
        return (f(tp) - f(tm)) / (2 * step)
    return (4 * cd(h / 2) - cd(h)) / 3 if richardson else cd(h)


def small_patch(seed=21, n_sources=3, n_bands=2, exp_per_band=2, size=40):
    from forcepho_b200 import synthetic as S
    p = S.config_multiband(seed=seed, render=O.render, n_sources=n_sources, n_bands=n_bands,
                           exp_per_band=exp_per_band, size=size)
    return p


def f32_theta(p, perturb=True, seed=3):
    th = p.scene.get_all_source_params().copy()
    nb = p.n_bands
    nper = nb + 6
    if perturb:
        rng = np.random.default_rng(seed)
        th = th.reshape(-1, nper)
        th[:, :nb] *= rng.uniform(0.9, 1.1, th[:, :nb].shape)
        th[:, nb] += rng.normal(0, 2e-6, len(th))
        th[:, nb + 1] += rng.normal(0, 2e-6, len(th))
        th[:, nb + 2] = np.clip(th[:, nb + 2] * 0.95, 0.3, 0.95)
        th[:, nb + 3] += 0.05
        th[:, nb + 4] = np.clip(th[:, nb + 4] + 0.1, 1.0, 5.0)
        th[:, nb + 5] = np.clip(th[:, nb + 5] * 1.05, 0.05, 0.5)
        th = th.reshape(-1)
    return th.astype(np.float32).astype(np.float64)


def oracle_chi2_total(p, th):
    p.scene.set_all_source_params(th)
    c, _, _ = O.evaluate(p, p.scene.get_proposal(), precision="f64")
    return float(np.sum(c))


def kinds(nb):
    return ["flux"] * nb + ["ra", "dec", "q", "pa", "sersic", "rhalf"]


def test_autograd_backward_vs_fd_and_reference():
    """Per parameter column, the backward pass against central differences of
    the FP64 oracle (power-of-two steps, exact in the f32 proposal) and against
    the reference CPU kernel's gradient; forward and backward run with no host
    synchronisation (torch's sync debug mode raises on one)."""
    import torch
    from forcepho_b200.autograd import PatchChi2
    from forcepho_b200.model import stack_grad
    p = small_patch()
    p.send_to_device()
    th = f32_theta(p)
    fn = PatchChi2(p)
    theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    torch.cuda.synchronize()
    torch.cuda.set_sync_debug_mode("error")
    try:
        chi2 = fn(theta)
        chi2.sum().backward()
    finally:
        torch.cuda.set_sync_debug_mode("default")
    assert chi2.shape == (p.n_bands,)
    g = theta.grad.cpu().numpy()

    # reference CPU kernel gradient at the same proposal
    p.scene.set_all_source_params(th)
    _, dref, _ = O.ref_evaluate(p, p.scene.get_proposal())
    gref = stack_grad(dref, int(p.n_sources), p.n_bands)

    # central differences of the FP64 oracle
    kk = kinds(p.n_bands) * int(p.n_sources)
    fd = np.zeros_like(th)
    for j, kind in enumerate(kk):
        fd[j] = central_difference(lambda t: oracle_chi2_total(p, t), th, j, FD_STEP[kind], kind in RICHARDSON)

    names = np.array(kk)
    achieved = {}
    for kind in FD_STEP:
        m = names == kind
        err_fd = np.linalg.norm(g[m] - fd[m]) / np.linalg.norm(fd[m])
        err_ref = np.linalg.norm(g[m] - gref[m]) / np.linalg.norm(gref[m])
        achieved[kind] = (err_fd, err_ref)
        assert err_ref < 1e-4, (kind, err_ref)
        assert err_fd < 1e-4, (kind, err_fd)
    print("per-column error vs FD of FP64 / vs reference kernel:",
          {k: ("%.1e" % a, "%.1e" % b) for k, (a, b) in achieved.items()})


def test_batched_autograd_matches_per_patch_and_replays_in_a_graph():
    """BatchChi2 over patches of different shapes equals PatchChi2 of each
    patch, forward and backward, bit for bit (the same kernels per tile and a
    fixed-order reduction); and its forward + vector-Jacobian product captured
    in a CUDA graph replays to the eager results at a new theta."""
    import torch
    from forcepho_b200.autograd import BatchChi2, PatchChi2
    rng = np.random.default_rng(4)
    patches = [small_patch(seed=int(rng.integers(1000)), n_sources=ns, n_bands=nb, size=36)
               for ns, nb in ((1, 1), (3, 2), (2, 3))]
    for p in patches:
        p.return_residual = False
        p.send_to_device()
    ths = [f32_theta(p, seed=i) for i, p in enumerate(patches)]
    f = BatchChi2(patches, tile_pixels=256)
    theta = torch.tensor(np.concatenate(ths), dtype=torch.float64, device="cuda", requires_grad=True)
    w = torch.linspace(0.5, 1.5, f.n_rows, dtype=torch.float64, device="cuda")
    chi2 = f(theta)
    (chi2 * w).sum().backward()
    gb = theta.grad.detach().clone()
    for i, p in enumerate(patches):
        fp = PatchChi2(p, tile_pixels=256)
        t1 = torch.tensor(ths[i], dtype=torch.float64, device="cuda", requires_grad=True)
        c1 = fp(t1)
        (c1 * w[f.band_slices[i]]).sum().backward()
        assert torch.equal(c1.detach(), chi2.detach()[f.band_slices[i]])
        assert torch.equal(t1.grad, gb[f.slices[i]])

    # graph capture of the device pieces: static theta in, chi2 and gradient out
    static_theta = theta.detach().clone()
    f._evaluate(static_theta)            # eager once: kernel attributes outside the capture
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        c_g, resp_g = f._evaluate(static_theta)
        g_g = f._vjp(w, resp_g)
    th2 = theta.detach() * (1 + 1e-3 * torch.cos(torch.arange(f.n_params, device="cuda", dtype=torch.float64)))
    static_theta.copy_(th2)
    graph.replay()
    torch.cuda.synchronize()
    t2 = th2.clone().requires_grad_(True)
    c_e = f(t2)
    (c_e * w).sum().backward()
    assert torch.equal(c_g, c_e.detach())
    assert torch.equal(g_g, t2.grad)


def make_hmc(n=3, seed=7, **kw):
    from forcepho_b200.hmc import DeviceHMC
    rng = np.random.default_rng(seed)
    patches = [small_patch(seed=int(rng.integers(1000)), n_sources=int(rng.integers(1, 4)), size=36)
               for _ in range(n)]
    for p in patches:
        p.return_residual = False
        p.send_to_device()
    theta = [f32_theta(p, seed=i) for i, p in enumerate(patches)]
    return DeviceHMC(patches, theta, **kw), patches, theta


def test_hmc_lnprob_matches_fastposterior():
    import torch
    from forcepho_b200.hmc import default_bounds
    from forcepho_b200.model import FastPosterior
    from forcepho_b200.proposal import B200Proposer
    h, patches, theta = make_hmc()
    h.gradient()
    torch.cuda.synchronize()
    z = h.z.cpu().numpy()
    lnp = h.lnp.cpu().numpy()
    grad = h.grad.cpu().numpy()
    for i, p in enumerate(patches):
        lo, hi = default_bounds(p, theta[i])
        post = FastPosterior(B200Proposer(), p, lower=lo, upper=hi)
        l, g = post.lnprob_and_grad(z[h.slices[i]])
        # host splines (scipy) and device splines round the f32 amplitudes
        # independently: agreement to f32 rounding of the proposal
        scale = float(np.sum((p.data.astype(np.float64) * p.ierr) ** 2))
        assert abs(l - lnp[i]) <= 1e-7 * scale, (i, l, lnp[i])
        gd = grad[h.slices[i]]
        assert np.linalg.norm(gd - g) <= 1e-5 * np.linalg.norm(g), (i, np.linalg.norm(gd - g) / np.linalg.norm(g))


def test_hmc_graph_equals_eager_and_conserves_energy():
    import torch
    h1, _, _ = make_hmc(seed=11, n_steps=4, max_traj=8, step_size=1e-3)
    h2, _, _ = make_hmc(seed=11, n_steps=4, max_traj=8, step_size=1e-3)
    h1.estimate_inv_mass()
    h2.inv_mass.copy_(h1.inv_mass)
    h1.run(3)                       # graph replays
    h2.gradient()
    for _ in range(3):              # eager launches
        h2._trajectory()
    torch.cuda.synchronize()
    assert torch.equal(h1.z, h2.z) and torch.equal(h1.lnp, h2.lnp)
    assert torch.equal(h1.accepted, h2.accepted)
    assert int(h1.traj.item()) == 3
    # tiny steps: leapfrog energy error far below 1
    assert float(h1.energy_error.abs().max()) < 1e-2
    assert int(h1.accepted.sum()) >= 1


def test_hmc_samples_move_and_accept():
    """Dual-averaging warm-up, then the averaged step sizes: chains move, and
    the mean acceptance probability after warm-up is near the target."""
    import torch
    h, _, _ = make_hmc(seed=13, n_steps=8, max_traj=60, step_size=0.05)
    h.estimate_inv_mass()
    z0 = h.z.clone()
    h.run(30, adapt=True, target=0.8)
    h.end_adaptation()
    torch.cuda.synchronize()
    assert torch.isfinite(h.lnp).all() and torch.isfinite(h.eps).all() and bool((h.eps > 0).all())
    acc = h.accepted.cpu().numpy()
    assert acc.min() >= 3, acc
    assert float((h.z - z0).abs().max()) > 0
    probs = []
    for _ in range(20):
        h.run(1)
        probs.append(torch.exp(torch.clamp(h.energy_error, max=0.0)).clone())
    mean_accept = float(torch.stack(probs).mean())
    assert 0.5 < mean_accept <= 1.0, mean_accept
