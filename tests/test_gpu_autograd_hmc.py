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
           "sersic": 2.0 ** -7, "rhalf": 2.0 ** -12}


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
    import torch
    from forcepho_b200.autograd import PatchChi2
    from forcepho_b200.model import stack_grad
    p = small_patch()
    p.send_to_device()
    th = f32_theta(p)
    fn = PatchChi2(p)
    theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    chi2 = fn(theta)
    assert chi2.shape == (p.n_bands,)
    chi2.sum().backward()
    g = theta.grad.cpu().numpy()

    # reference CPU kernel gradient at the same proposal
    p.scene.set_all_source_params(th)
    _, dref, _ = O.ref_evaluate(p, p.scene.get_proposal())
    gref = stack_grad(dref, int(p.n_sources), p.n_bands)

    # central differences of the FP64 oracle
    kk = kinds(p.n_bands) * int(p.n_sources)
    fd = np.zeros_like(th)
    for j, kind in enumerate(kk):
        h = FD_STEP[kind]
        tp, tm = th.copy(), th.copy()
        tp[j] += h
        tm[j] -= h
        fd[j] = (oracle_chi2_total(p, tp) - oracle_chi2_total(p, tm)) / (2 * h)

    names = np.array(kk)
    for kind in FD_STEP:
        m = names == kind
        err_fd = np.linalg.norm(g[m] - fd[m]) / np.linalg.norm(fd[m])
        err_ref = np.linalg.norm(g[m] - gref[m]) / np.linalg.norm(gref[m])
        assert err_ref < 1e-4, (kind, err_ref)
        assert err_fd < 2e-3, (kind, err_fd)


def test_autograd_any_band_function():
    """backward of a weighted sum of band chi2s uses the per-band Jacobian."""
    import torch
    from forcepho_b200.autograd import PatchChi2
    p = small_patch(seed=5)
    p.send_to_device()
    th = f32_theta(p, seed=9)
    fn = PatchChi2(p)
    w = torch.tensor([0.3, 1.7], dtype=torch.float64, device="cuda")
    theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    (fn(theta) * w).sum().backward()
    g = theta.grad.cpu().numpy()
    theta2 = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    c = fn(theta2)
    (0.3 * c[0]).backward()
    g0 = theta2.grad.cpu().numpy().copy()
    theta3 = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    (1.7 * fn(theta3)[1]).backward()
    g1 = theta3.grad.cpu().numpy()
    np.testing.assert_allclose(g, g0 + g1, rtol=1e-12, atol=1e-12 * np.abs(g).max())


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
    import torch
    h, _, _ = make_hmc(seed=13, n_steps=8, max_traj=40, step_size=0.05)
    h.estimate_inv_mass()
    z0 = h.z.clone()
    h.run(30, adapt=True)
    torch.cuda.synchronize()
    assert torch.isfinite(h.lnp).all()
    acc = h.accepted.cpu().numpy()
    assert acc.min() >= 3, acc
    assert float((h.z - z0).abs().max()) > 0
