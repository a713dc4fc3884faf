"""chi2 as a differentiable torch function of the scene parameters, on the device.

``BatchChi2(patches)`` maps the flat scene-parameter vector theta of many
device patches (per patch, per active source, the reference's order
``[flux_1..flux_nb, ra, dec, q, pa, sersic, rhalf]``, forcepho/sources.py:559-605)
to the per-band chi2 of every patch, concatenated patch by patch:

    f = BatchChi2(patches)
    chi2 = f(theta)                          # float64[sum of n_bands]
    (-0.5 * chi2.sum()).backward()           # theta.grad = dlnlike/dtheta

``PatchChi2(patch)`` is the one-patch form (chi2 float64[n_bands]).

Everything stays on the GPU, with no host synchronisation in forward or
backward, so both can be captured in a CUDA graph:

* forward: the proposal records are built on the device from theta
  (``fp_hmc_prepare``: the Sersic mixture amplitudes and their sersic / rhalf
  derivatives from the device B-spline tables), then one batched evaluation
  (``fp_evaluate_batch``: Gaussian setup, the persistent tile kernel with its
  hand-written adjoint, the fixed-order reduction) gives chi2 and every
  d chi2[band] / d(source parameter) in one pass; the Response records are
  kept for backward;
* backward: the vector-Jacobian product with those per-band derivatives,
  assembled like ``stack_grad`` (forcepho/model.py:370-387) but kept per band,
  so any function of the band chi2s differentiates correctly: a band's flux
  moves only that band's chi2, the six shape parameters move every band's.
"""

import ctypes

import numpy as np
import torch

from . import _native as N
from .device import Plan, current_stream_ptr, to_device_bytes
from .kernel_limits import MAXBANDS, MAXSOURCES, NPARAMS

__all__ = ["BatchChi2", "PatchChi2"]


class _Chi2Fn(torch.autograd.Function):

    @staticmethod
    def forward(ctx, theta, owner):
        chi2, resp = owner._evaluate(theta.detach())
        ctx.owner = owner
        ctx.theta_meta = (theta.device, theta.dtype)
        ctx.save_for_backward(resp)
        return chi2

    @staticmethod
    def backward(ctx, grad_chi2):
        (resp,) = ctx.saved_tensors
        dev, dt = ctx.theta_meta
        g = ctx.owner._vjp(grad_chi2.to(ctx.owner.device), resp)
        return g.to(device=dev, dtype=dt), None


class BatchChi2(torch.nn.Module):
    """Per-band chi2 of many device patches as one differentiable function.

    Parameters
    ----------
    patches : device patches (``send_to_device``-ed, B200PatchMixin)
    tile_pixels, ctas_per_sm : launch parameters of the tile kernel
    splines : the Sersic amplitude splines (default: the package's table)
    """

    def __init__(self, patches, tile_pixels=1024, ctas_per_sm=4, splines=None):
        super().__init__()
        from .hmc import spline_table
        self.L = N.load()
        self.patches = list(patches)
        self.n = len(self.patches)
        self.plan = Plan(self.patches, tile_pixels=tile_pixels)
        self.launch = self.plan.launch(ctas_per_sm=ctas_per_sm)
        dev = self.plan.device
        self.device = dev
        hp = np.zeros(self.n, dtype=N.hmc_patch_dtype)
        rows, flux_idx, shape_idx = [], [], []
        off = 0
        self.slices, self.band_slices = [], []
        nrow = 0
        for i, p in enumerate(self.patches):
            ns, nb = int(p.n_sources), int(p.n_bands)
            nper = nb + NPARAMS - 1
            hp[i] = (off, ns, nb)
            self.slices.append(slice(off, off + ns * nper))
            self.band_slices.append(slice(nrow, nrow + nb))
            rows += [i * MAXBANDS + b for b in range(nb)]
            for s in range(ns):
                for k in range(nper):
                    j = off + s * nper + k
                    if k < nb:      # flux in band k: Response[i, k, s, 0]
                        flux_idx.append((j, ((i * MAXBANDS + k) * MAXSOURCES + s) * NPARAMS))
                    else:           # shape parameter k - nb: column 1 + (k - nb) of every band
                        shape_idx.append((j, (i * MAXSOURCES + s) * (NPARAMS - 1) + (k - nb)))
            off += ns * nper
            nrow += nb
        self.n_params = off
        self.n_rows = nrow
        self.d_hp = to_device_bytes(hp, dev)
        i64 = dict(dtype=torch.int64, device=dev)
        self._rows = torch.tensor(rows, **i64)
        fi = np.array(flux_idx, np.int64).reshape(-1, 2)
        si = np.array(shape_idx, np.int64).reshape(-1, 2)
        self._flux_param, self._flux_src = torch.tensor(fi[:, 0], **i64), torch.tensor(fi[:, 1], **i64)
        self._shape_param, self._shape_src = torch.tensor(si[:, 0], **i64), torch.tensor(si[:, 1], **i64)
        self._theta_buf = torch.zeros(max(off, 1), dtype=torch.float64, device=dev)
        self._jac_buf = torch.zeros(max(off, 1), dtype=torch.float64, device=dev)
        self.tab = spline_table(dev, splines)
        self.ncall = 0

    def _evaluate(self, theta):
        """Queue proposal construction and one evaluation at theta; returns
        (chi2 rows, a copy of the Response records)."""
        if theta.shape != (self.n_params,):
            raise ValueError("theta has shape %s, expected (%d,)" % (tuple(theta.shape), self.n_params))
        th = theta.to(device=self.device, dtype=torch.float64).contiguous()
        s = current_stream_ptr()
        N.check(self.L.fp_hmc_prepare(self.d_hp.data_ptr(), self.n, th.data_ptr(), None, None,
                                      ctypes.byref(self.tab), self.plan.proposals.data_ptr(),
                                      self._theta_buf.data_ptr(), self._jac_buf.data_ptr(), s), "fp_hmc_prepare")
        self.plan.evaluate(self.launch)
        self.ncall += 1
        chi2 = self.plan.chi2.view(-1).index_select(0, self._rows)
        return chi2, self.plan.response.clone()

    def _vjp(self, grad_chi2, resp):
        """theta gradient of sum_rows grad_chi2[row] * chi2[row]."""
        g2 = torch.zeros(self.n * MAXBANDS, dtype=torch.float64, device=self.device)
        g2.index_copy_(0, self._rows, grad_chi2.to(torch.float64))
        r = resp.view(self.n, MAXBANDS, MAXSOURCES, NPARAMS)
        out = torch.zeros(self.n_params, dtype=torch.float64, device=self.device)
        # fluxes: one band each
        fl = r.reshape(-1).index_select(0, self._flux_src).to(torch.float64)
        out.index_copy_(0, self._flux_param, fl * g2.index_select(0, self._flux_src // (MAXSOURCES * NPARAMS)))
        # shape parameters: summed over the bands with their weights
        # (elementwise products and a sum: no library GEMM, so no handle or
        # workspace to create inside a graph capture)
        w = (g2.view(self.n, MAXBANDS, 1, 1) * r[..., 1:].to(torch.float64)).sum(dim=1)
        out.index_copy_(0, self._shape_param, w.reshape(-1).index_select(0, self._shape_src))
        return out

    def forward(self, theta):
        return _Chi2Fn.apply(theta, self)

    def split(self, chi2):
        """Per-patch views of a chi2 row vector."""
        return [chi2[sl] for sl in self.band_slices]


class PatchChi2(BatchChi2):
    """Per-band chi2 of one device patch as a torch function of theta
    (float64[n_sources * (n_bands + 6)] -> float64[n_bands])."""

    def __init__(self, patch, tile_pixels=None, ctas_per_sm=4, splines=None):
        if tile_pixels is None:
            from .autotune import default_tile_pixels
            tile_pixels = default_tile_pixels(patch)
        super().__init__([patch], tile_pixels=tile_pixels, ctas_per_sm=ctas_per_sm, splines=splines)
        self.patch = patch
        self.scene = getattr(patch, "scene", None)
        self.n_sources = int(patch.n_sources)
        self.n_bands = patch.n_bands
