"""The host posterior (forcepho_b200/model.py, after forcepho/model.py:260-637)
on the CPU, with the FP64 oracle standing in for the device proposer:

* ``BoundedTransform``: inverse round trip; Jacobian and d log|J|/dz against
  central differences;
* ``stack_grad``: the reference's parameter order [flux_1..flux_nb, ra, dec,
  q, pa, sersic, rhalf] per source, shape terms summed over bands;
* ``FastPosterior``: lnp = -chi2/2 + log|J| and its gradient through the
  transform, the Sersic-amplitude splines and the proposal, against central
  differences of lnp; the position cache;
* ``optimize_one_band``: the weighted linear flux solve.
"""

import numpy as np
import pytest

from oracle import oracle as O


class OracleProposer:
    """The proposer surface (``evaluate_proposal``) over the FP64 oracle."""

    def __init__(self):
        self.calls = 0

    def evaluate_proposal(self, proposal, patch=None, verbose=False, unpack=True):
        self.calls += 1
        chi2, dchi2, res = O.evaluate(patch, proposal, precision="f64", return_residual=patch.return_residual)
        return (chi2, dchi2, res) if patch.return_residual else (chi2, dchi2)


def test_bounded_transform_round_trip_and_jacobians():
    from forcepho_b200.model import BoundedTransform
    lo = np.array([0.0, -1.0, 0.2, 0.81])
    hi = np.array([10.0, 1.0, 1.0, 6.19])
    t = BoundedTransform(lo, hi)
    z = np.array([0.3, -1.2, 2.0, -0.4])
    q = t.transform(z)
    assert np.all((q > lo) & (q < hi))
    np.testing.assert_allclose(t.inverse_transform(q), z, rtol=1e-12, atol=1e-12)
    h = 1e-6
    jac_fd = np.array([(t.transform(z + h * e) - t.transform(z - h * e))[i] / (2 * h)
                       for i, e in enumerate(np.eye(len(z)))])
    np.testing.assert_allclose(t.jacobian(z), jac_fd, rtol=1e-7)
    ldj_fd = np.array([(t.lndetjac(z + h * e) - t.lndetjac(z - h * e)) / (2 * h) for e in np.eye(len(z))])
    np.testing.assert_allclose(t.lndetjac_grad(z), ldj_fd, rtol=1e-6, atol=1e-9)


def test_stack_grad_order():
    from forcepho_b200.model import stack_grad
    rng = np.random.default_rng(3)
    ns, nb = 3, 4
    d = rng.normal(size=(nb, ns, 7))
    g = stack_grad(d, ns, nb).reshape(ns, nb + 6)
    for s in range(ns):
        for b in range(nb):
            assert g[s, b] == d[b, s, 0]
        np.testing.assert_allclose(g[s, nb:], d[:, s, 1:].sum(axis=0), rtol=1e-15)


def _posterior():
    from forcepho_b200 import synthetic as S
    from forcepho_b200.hmc import default_bounds
    from forcepho_b200.model import FastPosterior
    p = S.config_multiband(seed=41, render=lambda pp, pr: O.render(pp, pr, precision="f64"), n_sources=2,
                           n_bands=2, exp_per_band=1, size=32, n_psf=2)
    p.return_residual = False
    theta = p.scene.get_all_source_params().copy()
    lo, hi = default_bounds(p, theta)
    post = FastPosterior(OracleProposer(), p, lower=lo, upper=hi)
    # a point off the truth, inside the bounds
    rng = np.random.default_rng(5)
    q0 = np.clip(theta + (hi - lo) * rng.uniform(-0.05, 0.05, theta.shape), lo + 1e-3 * (hi - lo),
                 hi - 1e-3 * (hi - lo))
    return post, post.transform.inverse_transform(q0)


def test_fastposterior_gradient_matches_central_differences():
    """The proposal records are float32 (as the reference's), so lnp carries
    rounding noise that central differences divide by the step: the error
    falls as 1/delta (1.7e-3 at 1e-5, 1.4e-4 at 1e-4, 1.5e-5 at 1e-3), and
    delta = 1e-3 in z keeps both it and the O(delta^2) term small."""
    post, z0 = _posterior()
    dlnp, num = post.check_grad(z0, delta=1e-3)
    assert np.all(np.isfinite(dlnp))
    err = np.linalg.norm(dlnp - num) / np.linalg.norm(num)
    assert err < 1e-4, err


def test_fastposterior_lnp_terms_and_cache():
    post, z0 = _posterior()
    lnp, grad = post.lnprob_and_grad(z0)
    n = post.proposer.calls
    lnp2, grad2 = post.lnprob_and_grad(z0.copy())       # same position: cached
    assert post.proposer.calls == n and lnp2 == lnp and np.array_equal(grad2, grad)
    q = post.transform.transform(z0)
    post.scene.set_all_source_params(q)
    chi2, _ = O.evaluate(post.patch, post.scene.get_proposal(), precision="f64")[:2]
    want = -0.5 * chi2.sum() + post.transform.lndetjac(z0)
    assert lnp == pytest.approx(want, rel=1e-12, abs=1e-9)


def test_optimize_one_band_recovers_fluxes():
    """The weighted flux solve (forcepho/fitting.py:572-587): noiseless data
    X^T f give back f, and the precision matrix is X_w X_w^T."""
    from forcepho_b200.fitting import optimize_one_band
    rng = np.random.default_rng(11)
    X = np.abs(rng.normal(size=(4, 300)))
    f = np.array([3.0, 0.5, 12.0, 7.0])
    w = rng.uniform(0.5, 2.0, 300)
    y = f @ X
    flux, prec = optimize_one_band(X, w, y)
    np.testing.assert_allclose(flux[:, 0], f, rtol=1e-10)
    np.testing.assert_allclose(prec, (X * w) @ (X * w).T, rtol=1e-12)
    # a fixed-source model is subtracted first
    flux2, _ = optimize_one_band(X, w, y + 2.0, fixedX=2.0)
    np.testing.assert_allclose(flux2[:, 0], f, rtol=1e-10)
