"""chi2 as a differentiable torch function of the scene parameters.

``PatchChi2(patch)`` maps the scene-parameter vector theta (the reference's
order: per active source ``[flux_1..flux_nb, ra, dec, q, pa, sersic, rhalf]``,
forcepho/sources.py:559-605) to the per-band chi2 vector, on the device:

    chi2 = PatchChi2(patch)(theta)           # float64[n_bands]
    (-0.5 * chi2.sum()).backward()           # theta.grad = dlnlike/dtheta

The forward pass runs the tiled sm_100a kernels, which compute chi2 and the
analytic gradient together (the hand-written adjoint); the backward pass is a
matrix-vector product of the upstream gradient with the saved per-band
Jacobian d chi2[b] / d theta, assembled like ``stack_grad``
(forcepho/model.py:370-387) but kept per band so any function of the band
chi2s differentiates correctly.  Sersic and rhalf derivatives flow through the
spline derivatives of the mixture amplitudes carried in the proposal.
"""

import numpy as np
import torch

from .kernel_limits import NPARAMS
from .proposal import B200Proposer

__all__ = ["PatchChi2", "chi2_jacobian"]


def chi2_jacobian(chi2_derivs, n_sources, n_bands):
    """(n_bands, n_sources, 7) kernel derivatives -> d chi2[b] / d theta,
    shape (n_bands, n_sources * (n_bands + 6))."""
    nper = n_bands + NPARAMS - 1
    J = np.zeros((n_bands, n_sources, nper), dtype=np.float64)
    d = np.asarray(chi2_derivs, dtype=np.float64)
    for b in range(n_bands):
        J[b, :, b] = d[b, :, 0]
        J[b, :, n_bands:] = d[b, :, 1:]
    return J.reshape(n_bands, n_sources * nper)


class _Chi2Fn(torch.autograd.Function):

    @staticmethod
    def forward(ctx, theta, owner):
        chi2, jac = owner._evaluate(theta.detach())
        ctx.save_for_backward(jac)
        return chi2

    @staticmethod
    def backward(ctx, grad_chi2):
        (jac,) = ctx.saved_tensors
        return grad_chi2.to(jac.dtype) @ jac, None


class PatchChi2(torch.nn.Module):
    """Per-band chi2 of one device patch as a torch function of theta.

    Parameters
    ----------
    patch : a device patch (``B200PatchMixin``) with a ``scene``
    proposer : defaults to ``B200Proposer()``
    """

    def __init__(self, patch, proposer=None):
        super().__init__()
        self.patch = patch
        self.scene = patch.scene
        self.proposer = proposer or B200Proposer()
        self.n_sources = int(patch.n_sources)
        self.n_bands = patch.n_bands
        self.ncall = 0

    @property
    def n_params(self):
        return self.n_sources * (self.n_bands + NPARAMS - 1)

    def _evaluate(self, theta):
        th = theta.detach().to("cpu", torch.float64).numpy()
        self.scene.set_all_source_params(th)
        chi2, derivs = self.proposer.evaluate_proposal(self.scene.get_proposal(), patch=self.patch)[:2]
        self.ncall += 1
        J = chi2_jacobian(derivs, self.n_sources, self.n_bands)
        dev = theta.device
        return (torch.from_numpy(np.asarray(chi2, np.float64)).to(dev),
                torch.from_numpy(J).to(dev))

    def forward(self, theta):
        if theta.shape != (self.n_params,):
            raise ValueError("theta has shape %s, expected (%d,)" % (tuple(theta.shape), self.n_params))
        return _Chi2Fn.apply(theta, self)
