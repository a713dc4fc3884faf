"""Posteriors over scene parameters: the consumers of lnlike and its gradient.

Mirrors forcepho/model.py so the reference's samplers and optimisers
(``fitting.run_lmc``'s ``logp_dlogp_func=model.lnprob_and_grad``,
``run_opt``'s ``model.nll``) can drive the B200 proposers unchanged:

* ``Posterior``      -- caching of lnp / grad by position, ``lnprob``,
  ``lnprob_grad``, ``lnprob_and_grad``, ``nll``, ``check_grad`` (central
  differences) (model.py:42-257);
* ``FastPosterior``  -- ``evaluate(z)``: transform to scene parameters, build
  the proposal, call ``proposer.evaluate_proposal``, lnlike = -chi2/2 summed
  in f64, gradient reordered by ``stack_grad`` (model.py:260-405);
* ``Transform`` / ``BoundedTransform`` -- identity and sigmoid maps with their
  diagonal Jacobians and log-determinant gradients (model.py:555-637).
"""

import numpy as np
from scipy.special import expit

from .kernel_limits import NPARAMS

__all__ = ["Posterior", "FastPosterior", "GPUPosterior", "Transform", "BoundedTransform", "stack_grad",
           "sigmoid", "logit", "sigmoid_grad"]


def stack_grad(chi2_derivs, n_sources, n_bands):
    """(n_bands, n_sources, 7) chi2 derivatives -> the scene-parameter order
    [flux_1..flux_nb, ra, dec, q, pa, sersic, rhalf] per source, shape
    parameters summed over bands (model.py:370-387)."""
    grads = np.zeros([n_sources, n_bands + (NPARAMS - 1)], dtype=np.float64)
    for band, derivs in enumerate(chi2_derivs):
        grads[:, n_bands:] += derivs[:, 1:]
        grads[:, band] += derivs[:, 0]
    return grads.reshape(-1)


class Posterior:
    """Caching base class (model.py:42-257)."""

    def __init__(self, transform=None, lower=None, upper=None):
        self.ncall = 0
        self.ndof = 1.0
        if (transform is None) == (lower is None or upper is None):
            raise ValueError('Must specify either "transform" or ("lower","upper")')
        self.transform = transform if transform is not None else BoundedTransform(lower, upper)
        self._z = -99
        self._lnpriorfn = None

    def evaluate(self, z):
        raise NotImplementedError

    def _stale(self, z):
        return np.shape(self._z) != np.shape(z) or np.any(z != self._z)

    def lnprob(self, z):
        if self._stale(z):
            self.evaluate(z)
        return self._lnp

    def lnprob_grad(self, z):
        if self._stale(z):
            self.evaluate(z)
        return self._lnp_grad

    def lnprob_and_grad(self, z):
        if self._stale(z):
            self.evaluate(z)
        return self._lnp, self._lnp_grad

    def nll(self, z):
        if self._stale(z):
            self.evaluate(z)
        return -self._lnp / self.ndof, -self._lnp_grad / self.ndof

    def nll_nograd(self, z):
        if self._stale(z):
            self.evaluate(z)
        return -self._lnp / self.ndof

    def lnprior(self, q):
        if self._lnpriorfn is None:
            return 0.0, 0.0
        return self._lnpriorfn(q)

    def make_transform(self, z):
        if self.transform is not None:
            self._jacobian = self.transform.jacobian(z)
            self._lndetjac = self.transform.lndetjac(z)
            self._lndetjac_grad = self.transform.lndetjac_grad(z)
            return self.transform.transform(z)
        self._jacobian, self._lndetjac, self._lndetjac_grad = 1.0, 0.0, 0.0
        return np.array(z)

    def check_grad(self, z, delta=1e-5):
        """Analytic and central-difference gradients of lnprob at z."""
        z0 = np.array(z, dtype=np.float64)
        dlnp = np.array(self.lnprob_grad(z0))
        delta = np.zeros_like(dlnp) + delta
        num = np.zeros(len(z0))
        for i, dp in enumerate(delta):
            t = z0.copy()
            t[i] -= dp
            lo = self.lnprob(t.copy())
            t[i] += 2 * dp
            hi = self.lnprob(t.copy())
            num[i] = (hi - lo) / (2 * dp)
        return dlnp, num


class FastPosterior(Posterior):
    """lnp(z) from a device proposer (model.py:260-368).

    Parameters
    ----------
    proposer : object with ``evaluate_proposal(proposal, patch=...)``
    patch    : the (device) patch
    scene    : the ``Scene`` whose active sources the parameters describe
    """

    def __init__(self, proposer, patch, scene=None, lnprior=None, transform=None, lower=None, upper=None,
                 sampling=True, logging=False):
        super().__init__(transform=transform, lower=lower, upper=upper)
        self.proposer = proposer
        self.patch = patch
        self.scene = scene if scene is not None else patch.scene
        self._lnpriorfn = lnprior
        self.sampling = sampling
        self.logging = logging
        self.mhalf = np.array(-0.5, dtype=np.float64)
        if logging:
            self.pos_history, self.lnp_history, self.grad_history = [], [], []

    def evaluate(self, z):
        q = self.make_transform(z)
        self.scene.set_all_source_params(q)
        proposal = self.scene.get_proposal()
        lpr, lpr_grad = self.lnprior(q)
        ret = self.proposer.evaluate_proposal(proposal, patch=self.patch)
        chi2, chi2_derivs = ret[0], ret[1]
        if len(ret) == 3:
            self._residuals = ret[2]
        ll = self.mhalf * np.array(chi2.astype(np.float64).sum(), dtype=np.float64)
        ll_grad = self.mhalf * self.stack_grad(chi2_derivs)
        self.ncall += 1
        self._lnlike, self._lnlike_grad = ll, ll_grad
        self._lnp = ll + lpr
        self._lnp_grad = (ll_grad + lpr_grad) * self._jacobian
        self._q, self._z = q, np.array(z)
        if self.sampling:
            self._lnp = self._lnp + self._lndetjac
            self._lnp_grad = self._lnp_grad + self._lndetjac_grad
        if self.logging:
            self.pos_history.append(np.array(z))
            self.lnp_history.append(ll)
            self.grad_history.append(ll_grad)

    def stack_grad(self, chi2_derivs):
        return stack_grad(chi2_derivs, int(self.patch.n_sources), self.patch.n_bands)

    def residuals(self, q, unpack=True):
        orig = self.patch.return_residual
        self.patch.return_residual = True
        self.scene.set_all_source_params(q)
        ret = self.proposer.evaluate_proposal(self.scene.get_proposal(), patch=self.patch, unpack=unpack)
        self.patch.return_residual = orig
        self._residuals = ret[2]
        return self._residuals


class GPUPosterior(FastPosterior):
    """The reference's backwards-compatible name for ``FastPosterior``
    (forcepho/model.py:408-411)."""


def sigmoid(x):
    return expit(x)


def logit(y):
    return -np.log(1.0 / y - 1.0)


def sigmoid_grad(z):
    """sigmoid(z) (1 - sigmoid(z)) in the overflow-safe form (0.5 / cosh(z/2))^2."""
    return (0.5 / np.cosh(0.5 * z)) ** 2


class Transform:
    """Identity transform (model.py:555-575)."""

    def __init__(self, ndim):
        self.ndim = ndim

    def transform(self, z):
        return np.array(z)

    def jacobian(self, z):
        return np.ones(len(z))

    def lndetjac(self, z):
        return float(np.log(np.abs(np.prod(self.jacobian(z)))))

    def lndetjac_grad(self, z):
        return np.zeros(len(z))

    def inverse_transform(self, q):
        return np.array(q)


class BoundedTransform(Transform):
    """q = lower + (upper - lower) sigmoid(z) (model.py:578-637).

    ``lndetjac`` is the sum of log(dq/dz) (computed directly, which equals the
    reference's log |prod J|); ``lndetjac_grad`` = 1 - 2 sigmoid(z)."""

    def __init__(self, lower, upper):
        self.lower = np.atleast_1d(np.asarray(lower, dtype=np.float64))
        self.upper = np.atleast_1d(np.asarray(upper, dtype=np.float64))
        if len(self.upper) != len(self.lower):
            raise ValueError("lower and upper differ in length")
        self.ndim = len(self.upper)

    @property
    def range(self):
        return self.upper - self.lower

    def transform(self, z):
        return self.lower + sigmoid(np.asarray(z, dtype=np.float64)) * self.range

    def jacobian(self, z):
        return self.range * sigmoid_grad(np.asarray(z, dtype=np.float64))

    def lndetjac(self, z):
        return float(np.sum(np.log(np.abs(self.jacobian(z)))))

    def lndetjac_grad(self, z):
        return 1.0 - 2.0 * sigmoid(np.asarray(z, dtype=np.float64))

    def inverse_transform(self, q):
        return logit((np.asarray(q, dtype=np.float64) - self.lower) / self.range)
