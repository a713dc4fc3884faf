"""Spline amplitudes: the device algorithm's host twin against scipy (CPU), and
the device proposal builder against Galaxy.proposal (GPU)."""

import numpy as np
import pytest

from forcepho_b200.splines import default_splines


def basis(t, n, k, x):
    """Host twin of bspline_basis in forcepho_b200/csrc/hmc.cu (same steps)."""
    x = min(max(x, t[k]), t[n])
    a, b = k, n - 1
    while a < b:
        m = (a + b + 1) >> 1
        if t[m] <= x:
            a = m
        else:
            b = m - 1
    l = a
    N = np.zeros(k + 1)
    left, right, lower = np.zeros(k + 1), np.zeros(k + 1), np.zeros(k + 1)
    N[0] = 1.0
    for j in range(1, k + 1):
        left[j] = x - t[l + 1 - j]
        right[j] = t[l + j] - x
        saved = 0.0
        for r in range(j):
            tmp = N[r] / (right[r + 1] + left[j - r])
            N[r] = saved + right[r + 1] * tmp
            saved = left[j - r] * tmp
        N[j] = saved
        if j == k - 1:
            lower[:j + 1] = N[:j + 1]
    dN = np.zeros(k + 1)
    for r in range(k + 1):
        i = l - k + r
        d = 0.0
        if r >= 1 and t[i + k] - t[i] > 0:
            d += lower[r - 1] / (t[i + k] - t[i])
        if r <= k - 1 and t[i + k + 1] - t[i + 1] > 0:
            d -= lower[r] / (t[i + k + 1] - t[i + 1])
        dN[r] = k * d
    return l - k, N, dN


def twin_eval(sp, x, y):
    tx, ty, c, kx, ky = sp.tck()
    ncx, ncy = len(tx) - kx - 1, len(ty) - ky - 1
    ix, Nx, dNx = basis(tx, ncx, kx, x)
    iy, Ny, dNy = basis(ty, ncy, ky, y)
    out = []
    for r in range(c.shape[0]):
        C = c[r].reshape(ncx, ncy)[ix:ix + kx + 1, iy:iy + ky + 1]
        out.append((Nx @ C @ Ny, dNx @ C @ Ny, Nx @ C @ dNy))
    return np.array(out)


@pytest.mark.parametrize("x,y", [(2.0, 0.15), (0.8, 0.0), (6.2, 1.0), (1.0, 0.02), (3.33, 0.517),
                                 (7.5, 1.3), (0.5, -0.1), (4.0, 0.03)])
def test_twin_matches_scipy(x, y):
    sp = default_splines()
    got = twin_eval(sp, x, y)
    want = np.array([[s(x, y)[0, 0], s(x, y, dx=1)[0, 0], s(x, y, dy=1)[0, 0]] for s in sp.splines])
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12)


def test_knots_shared():
    tx, ty, c, kx, ky = default_splines().tck()
    assert (kx, ky) == (3, 3) and c.shape == (9, 55 * 101)


@pytest.mark.gpu
def test_device_proposals_match_host():
    import torch
    from forcepho_b200 import synthetic as S
    from forcepho_b200.hmc import DeviceHMC
    rng = np.random.default_rng(5)
    patches = [S.config_multiband(seed=int(rng.integers(1000)), n_sources=5, n_bands=2, exp_per_band=1, size=40)
               for _ in range(3)]
    for p in patches:
        p.send_to_device()
    theta = [p.scene.get_all_source_params() for p in patches]
    h = DeviceHMC(patches, theta)
    th = h.positions()
    torch.cuda.synchronize()
    dev = h.proposals()
    for i, p in enumerate(patches):
        p.scene.set_all_source_params(th[i])
        host = p.scene.get_proposal()
        ns = int(p.n_sources)
        for f in ["ra", "dec", "q", "pa", "nsersic", "rh"]:
            np.testing.assert_allclose(dev[i][f][:ns], host[f], rtol=2e-7, atol=1e-12)
        for f in ["fluxes", "mixture_amplitudes", "damplitude_drh", "damplitude_dnsersic"]:
            np.testing.assert_allclose(dev[i][f][:ns], host[f], rtol=2e-6, atol=2e-7 * np.abs(host[f]).max())
