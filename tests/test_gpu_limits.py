"""The limits workload on the GPU: 30 sources, 8 bands x 4 exposures of
256x256 pixels, 6-Gaussian PSFs (1620 image Gaussians per exposure, 2.1 M
pixels).  The CPU checkers are run on a subset of bands (each band is an
independent output of the kernel), which keeps them to seconds."""

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import CHI2_F64, CHI2_REF, GRAD_F64, GRAD_REF, RAW_FLOOR, grad_err, ref_gap_explained

pytestmark = pytest.mark.gpu

BANDS = (0, 5)


@pytest.fixture(scope="module")
def limits_patch():
    from forcepho_b200 import synthetic as S
    from forcepho_b200.batch import render_models
    p = S.config_limits(seed=3)
    rng = np.random.default_rng(31)
    model = render_models([p])[0]
    S.add_noise(p, rng, rng.uniform(0.5, 2.0, p.n_exp), model)
    p.return_residual = True
    p.send_to_device()
    th = p.scene.get_all_source_params().reshape(30, -1)
    th[:, 8] *= 1.0 + rng.normal(0, 1e-7, 30)            # ra, dec off the truth
    th[:, 9] += rng.normal(0, 1e-6, 30)
    th[:, 10] = np.clip(th[:, 10] * 0.97, 0.2, 0.99)      # q
    p.scene.set_all_source_params(th.reshape(-1))
    return p, p.scene.get_proposal().copy()


def band_scale(p, res, b):
    e0, ne = int(p.band_start[b]), int(p.band_N[b])
    s0 = int(p.exposure_start[e0])
    s1 = int(p.exposure_start[e0 + ne - 1] + p.exposure_N[e0 + ne - 1])
    d = p.data[s0:s1].astype(np.float64) * p.ierr[s0:s1]
    r = np.asarray(res[s0:s1], np.float64) * p.ierr[s0:s1]
    return float(np.sum(d * d + r * r))


@pytest.mark.parametrize("kind", ["tiled", "plain"])
def test_limits_parity(limits_patch, kind):
    from forcepho_b200.proposal import B200Proposer, PlainProposer
    p, prop = limits_patch
    assert p.max_gauss_per_exposure() == 1620 and p.npix == 32 * 65536
    chi2, dchi2, res = (B200Proposer() if kind == "tiled" else PlainProposer()).evaluate_proposal(
        prop, patch=p, unpack=False)
    c64, g64, _ = O.evaluate(p, prop, precision="f64", bands=BANDS)
    cref, gref, _ = O.ref_evaluate(p, prop, bands=BANDS)
    tol_c, tol_g = (CHI2_F64, GRAD_F64) if kind == "tiled" else (CHI2_REF, GRAD_REF)
    for b in BANDS:
        sc = band_scale(p, res, b)
        raw64 = abs(chi2[b] - c64[b]) / max(abs(c64[b]), RAW_FLOOR * sc)
        eref = abs(chi2[b] - cref[b]) / sc
        g64e = grad_err(dchi2[b], g64[b])
        grefe = grad_err(dchi2[b], gref[b])
        assert eref < CHI2_REF and grefe < GRAD_REF, (kind, b, eref, grefe)
        assert raw64 < tol_c and g64e < tol_g, (kind, b, raw64, g64e)
        assert ref_gap_explained(chi2[b], cref[b], c64[b], tol_c, sc), (kind, b, chi2[b], cref[b], c64[b])


def test_limits_autograd_and_fd(limits_patch):
    """PatchChi2 at 420 parameters; backward against central differences of
    the FP64 oracle's chi2 of one band, for every parameter of two sources."""
    import torch
    from forcepho_b200.autograd import PatchChi2
    p, prop = limits_patch
    p.return_residual = False
    th0 = p.scene.get_all_source_params().astype(np.float32).astype(np.float64)
    fn = PatchChi2(p)
    theta = torch.tensor(th0, dtype=torch.float64, device="cuda", requires_grad=True)
    w = torch.zeros(p.n_bands, dtype=torch.float64, device="cuda")
    b = BANDS[1]
    w[b] = 1.0
    (fn(theta) * w).sum().backward()
    g = theta.grad.cpu().numpy().reshape(30, 14)
    from test_gpu_autograd_hmc import FD_STEP, RICHARDSON, central_difference
    kinds = ["flux", "ra", "dec", "q", "pa", "sersic", "rhalf"]

    def chi2_b(th):
        p.scene.set_all_source_params(th)
        return O.evaluate(p, p.scene.get_proposal(), precision="f64", bands=[b])[0][b]

    cols = [b] + list(range(8, 14))         # this band's flux, then ra..rhalf
    srcs = (3, 17, 25)
    fd = np.zeros((len(srcs), len(cols)))
    for i, s in enumerate(srcs):
        for k, col in enumerate(cols):
            fd[i, k] = central_difference(chi2_b, th0, s * 14 + col, FD_STEP[kinds[k]], kinds[k] in RICHARDSON)
    p.scene.set_all_source_params(th0)
    an = g[list(srcs)][:, cols]
    # per parameter column, normwise over the sources; and each component
    # within 1e-4 of its column's norm (the finite differences' own noise
    # is about 1e-5 of that)
    for k in range(len(cols)):
        den = np.linalg.norm(fd[:, k])
        assert np.linalg.norm(an[:, k] - fd[:, k]) <= 1e-4 * den, (kinds[k], an[:, k], fd[:, k])
        assert np.all(np.abs(an[:, k] - fd[:, k]) <= 1e-4 * den), (kinds[k], an[:, k], fd[:, k])
