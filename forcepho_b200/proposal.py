"""Proposers: the host boundary of the likelihood kernels.

``B200Proposer`` is a drop-in for the reference's ``GPUProposer``
(forcepho/proposal.py:55-152): ``evaluate_proposal(proposal, patch=None,
verbose=False, unpack=True)`` takes a ``source_struct_dtype`` array and a patch
that has been ``send_to_device``-ed, and returns

* ``chi2``        float64[n_bands]
* ``chi2_derivs`` float32[n_bands, n_sources, 7] (dflux, dra, ddec, dq, dpa,
  dsersic, drh), a view of the Response records as the reference makes it
* ``residuals``   list of per-exposure arrays (or the flat array with
  ``unpack=False``) -- only when ``patch.return_residual``.

It runs the tiled sm_100a kernels through the C ABI (``fp_evaluate_batch`` with
one patch).  ``PlainProposer`` has the same surface over the one-CTA-per-band
comparator kernel (``fp_evaluate_proposal_plain``), and ``F64Proposer`` the
FP64 device evaluation (``fp_evaluate_proposal_f64``, a precision reference
without residuals).  ``Proposer`` is an alias
of ``B200Proposer``, as ``Proposer`` aliases ``GPUProposer`` in the reference.
"""

import ctypes
import sys

import numpy as np
import torch

from . import _native as N
from .device import Plan, current_stream_ptr, response_view
from .kernel_limits import MAXBANDS, MAXRADII, MAXSOURCES, NPARAMS
from .structs import response_struct_dtype, source_struct_dtype

__all__ = ["ProposerBase", "B200Proposer", "PlainProposer", "F64Proposer", "Proposer",
           "source_struct_dtype", "response_struct_dtype", "MAXBANDS", "MAXRADII", "MAXSOURCES", "NPARAMS"]


class ProposerBase:

    def evaluate_proposal(self, proposal, **kwargs):
        raise NotImplementedError

    def unpack_residuals(self, residuals_flat, patch, reshape=False):
        """Split the flat padded residual into per-exposure arrays; with
        ``reshape`` drop the padding and reshape to the original stamps
        (forcepho/proposal.py:38-52)."""
        residuals = np.split(residuals_flat, np.cumsum(patch.exposure_N)[:-1])
        if reshape:
            for e, r in enumerate(residuals):
                r = r[:patch.original_sizes[e]]
                residuals[e] = r.reshape(patch.original_shapes[e])
        return residuals

    @staticmethod
    def _check_proposal(proposal, patch):
        p = np.ascontiguousarray(proposal)
        if p.dtype != source_struct_dtype:
            p = p.astype(source_struct_dtype)
        p = p.reshape(-1)
        if len(p) != int(patch.n_sources):
            raise ValueError("proposal has %d sources, the patch %d" % (len(p), int(patch.n_sources)))
        return p

    @staticmethod
    def _ensure_residual(patch):
        if patch.return_residual and "residual" not in patch.device_ptrs:
            patch._alloc_residual()
            patch.send_patchstruct_to_device()


class B200Proposer(ProposerBase):
    """Evaluate proposals on one device patch with the tiled sm_100a kernels.

    Parameters
    ----------
    patch : optional default patch (as in the reference).
    tile_pixels : pixel-tile size of the work plan (256, 512 or 1024), or None
        for the autotuned default of the patch's size class.
    ctas_per_sm : persistent CTAs per SM.
    flags : extra ``fp_launch`` flags (e.g. ``FLAG_NO_CULL``).
    use_graph : replay the proposal upload, the three launches and the read-back
        of a plan as one CUDA graph (captured on the plan's first call); False
        issues them one by one.
    """

    def __init__(self, patch=None, tile_pixels=None, ctas_per_sm=4, flags=0, use_graph=True):
        N.load()
        self.patch = patch
        self.tile_pixels = tile_pixels
        self.ctas_per_sm = ctas_per_sm
        self.flags = flags
        self.use_graph = use_graph
        self._plan = None
        self._plan_key = None
        self._pinned_prop = None
        self._pinned_out = None
        self._graph = None
        self._graph_key = None

    def plan_for(self, patch):
        key = (id(patch), patch.plan_signature(), self.tile_pixels)
        if self._plan is None or self._plan_key != key:
            tp = self.tile_pixels
            if tp is None:
                from .autotune import default_tile_pixels
                tp = default_tile_pixels(patch)
            self._graph = None              # captured over the previous plan's buffers
            self._plan = Plan([patch], tile_pixels=tp)
            self._plan_key = key
            self._pinned_prop = torch.zeros(self._plan.proposals.numel(), dtype=torch.uint8).pin_memory()
            self._pinned_chi2 = torch.zeros((1, MAXBANDS), dtype=torch.float64).pin_memory()
            self._pinned_resp = torch.zeros((1, MAXBANDS, MAXSOURCES * NPARAMS), dtype=torch.float32).pin_memory()
        return self._plan

    def evaluate_proposal(self, proposal, patch=None, verbose=False, unpack=True):
        if patch is None:
            patch = self.patch
        prop = self._check_proposal(proposal, patch)
        self._ensure_residual(patch)
        plan = self.plan_for(patch)
        n_bands, n_sources = patch.n_bands, int(patch.n_sources)
        if verbose:
            print("Launching tiled evaluation: %d tiles of %d px, %d CTAs/SM"
                  % (plan.sizes.n_tiles, plan.tile_pixels, self.ctas_per_sm), file=sys.stderr, flush=True)
        self._pinned_prop.numpy()[:prop.nbytes] = prop.view(np.uint8)     # n_sources records
        stream = torch.cuda.current_stream()
        lp = plan.launch(ctas_per_sm=self.ctas_per_sm, flags=self.flags)
        if self.use_graph:
            gkey = (self._plan_key, self.ctas_per_sm, self.flags)
            if self._graph is None or self._graph_key != gkey:
                self._capture(plan, lp, stream)
                self._graph_key = gkey
            plan.check_current(stream)
            self._graph.replay()
        else:
            self._queue(plan, lp)
        stream.synchronize()
        chi_out = self._pinned_chi2.numpy()[0, :n_bands].copy()
        chi_derivs = response_view(self._pinned_resp.numpy()[0], n_bands, n_sources).copy()
        if patch.return_residual:
            residuals = patch.retrieve_array("residual")
            if unpack:
                residuals = self.unpack_residuals(residuals, patch)
            return chi_out, chi_derivs, residuals
        return chi_out, chi_derivs

    def _queue(self, plan, lp):
        """Proposal upload, evaluation and read-back on the current stream:
        only the plan's source records and the patch's band rows cross PCIe
        (the kernels read n_sources records and write n_bands rows)."""
        patch = plan.patches[0]
        nrec = int(patch.n_sources) * source_struct_dtype.itemsize
        nb = patch.n_bands
        if nrec:
            plan.proposals[:nrec].copy_(self._pinned_prop[:nrec], non_blocking=True)
        plan.evaluate(lp)
        self._pinned_chi2[0, :nb].copy_(plan.chi2[0, :nb], non_blocking=True)
        self._pinned_resp[0, :nb].copy_(plan.response[0, :nb], non_blocking=True)

    def _capture(self, plan, lp, stream):
        # one eager pass first sets the kernels' attributes outside the capture
        self._queue(plan, lp)
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._queue(plan, lp)
        torch.cuda.synchronize()
        self._graph = g


class F64Proposer(ProposerBase):
    """The likelihood and gradient of one proposal in FP64 on the device
    (``fp_evaluate_proposal_f64``): a precision reference for whole patches,
    where the CPU oracle is too slow.  ``evaluate_proposal`` returns

    * ``chi2``        float64[n_bands]
    * ``chi2_derivs`` float64[n_bands, n_sources, 7], same order as the
      Response records.

    No residual is written and nothing is culled; a patch whose exposures
    hold more Gaussians than the plan raises ``RuntimeError``.
    """

    def __init__(self, patch=None):
        self.L = N.load()
        self.patch = patch
        self._ws = None

    def _workspace(self, patch, max_gauss, device):
        n = ctypes.c_size_t()
        N.check(self.L.fp_f64_workspace_bytes(patch.n_exp, max_gauss, ctypes.byref(n)), "fp_f64_workspace_bytes")
        if self._ws is None or self._ws.numel() < n.value or self._ws.device != device:
            self._ws = torch.zeros(n.value, dtype=torch.uint8, device=device)
        return self._ws, n.value

    def evaluate_proposal(self, proposal, patch=None, verbose=False, unpack=True):
        if patch is None:
            patch = self.patch
        prop = self._check_proposal(proposal, patch)
        device = patch.device_patch.device
        n_bands, n_sources = patch.n_bands, int(patch.n_sources)
        max_gauss = patch.max_gauss_per_exposure()
        ws, nbytes = self._workspace(patch, max_gauss, device)
        host = np.zeros(max(len(prop), 1), dtype=source_struct_dtype)
        host[:len(prop)] = prop
        d_prop = torch.from_numpy(host.view(np.uint8).copy()).to(device)
        chi2 = torch.zeros(MAXBANDS, dtype=torch.float64, device=device)
        dchi2 = torch.zeros((MAXBANDS, MAXSOURCES, NPARAMS), dtype=torch.float64, device=device)
        stream = torch.cuda.current_stream()
        if verbose:
            print("Launching FP64 evaluation over %d exposures" % patch.n_exp, file=sys.stderr, flush=True)
        N.check(self.L.fp_evaluate_proposal_f64(
            ctypes.c_void_p(patch.device_patch_ptr), ctypes.c_void_p(d_prop.data_ptr()), n_bands, patch.n_exp,
            max_gauss, ctypes.c_void_p(chi2.data_ptr()), ctypes.c_void_p(dchi2.data_ptr()),
            ctypes.c_void_p(ws.data_ptr()), nbytes, current_stream_ptr(stream)), "fp_evaluate_proposal_f64")
        st = ctypes.c_int32()
        N.check(self.L.fp_read_status(ctypes.c_void_p(ws.data_ptr()), ctypes.byref(st), current_stream_ptr(stream)),
                "fp_read_status")
        if st.value:
            raise RuntimeError("fp_evaluate_proposal_f64: device status %d" % st.value)
        out_chi2 = chi2[:n_bands].cpu().numpy()
        out_d = dchi2[:n_bands, :n_sources].cpu().numpy()
        return out_chi2, out_d


Proposer = B200Proposer


class PlainProposer(ProposerBase):
    """Same surface, evaluated by the port-equivalent kernel: one 1024-thread
    CTA per band and one launch per patch (the comparator)."""

    def __init__(self, patch=None):
        self.L = N.load()
        self.patch = patch
        self._bufs = None

    def _buffers(self, device):
        if self._bufs is None:
            self._bufs = dict(
                prop=torch.zeros(MAXSOURCES * source_struct_dtype.itemsize, dtype=torch.uint8, device=device),
                chi2=torch.zeros(MAXBANDS, dtype=torch.float64, device=device),
                resp=torch.zeros((MAXBANDS, MAXSOURCES * NPARAMS), dtype=torch.float32, device=device),
                pin_prop=torch.zeros(MAXSOURCES * source_struct_dtype.itemsize, dtype=torch.uint8).pin_memory(),
                pin_chi2=torch.zeros(MAXBANDS, dtype=torch.float64).pin_memory(),
                pin_resp=torch.zeros((MAXBANDS, MAXSOURCES * NPARAMS), dtype=torch.float32).pin_memory())
        return self._bufs

    def launch(self, patch, d_proposal_ptr, d_chi2_ptr, d_resp_ptr, stream=None):
        """Queue one plain evaluation (device pointers; no host synchronisation)."""
        N.check(self.L.fp_evaluate_proposal_plain(
            ctypes.c_void_p(patch.device_patch_ptr), ctypes.c_void_p(d_proposal_ptr), patch.n_bands,
            patch.max_gauss_per_exposure(), ctypes.c_void_p(d_chi2_ptr), ctypes.c_void_p(d_resp_ptr),
            current_stream_ptr(stream)), "fp_evaluate_proposal_plain")

    def evaluate_proposal(self, proposal, patch=None, verbose=False, unpack=True):
        if patch is None:
            patch = self.patch
        prop = self._check_proposal(proposal, patch)
        self._ensure_residual(patch)
        b = self._buffers(patch.device_patch.device)
        n_bands, n_sources = patch.n_bands, int(patch.n_sources)
        host = np.zeros(MAXSOURCES, dtype=source_struct_dtype)
        host[:len(prop)] = prop
        b["pin_prop"].numpy()[:] = host.view(np.uint8)
        stream = torch.cuda.current_stream()
        b["prop"].copy_(b["pin_prop"], non_blocking=True)
        if verbose:
            print("Launching plain kernel with grid (%d,), block 1024" % n_bands, file=sys.stderr, flush=True)
        self.launch(patch, b["prop"].data_ptr(), b["chi2"].data_ptr(), b["resp"].data_ptr(), stream)
        b["pin_chi2"].copy_(b["chi2"], non_blocking=True)
        b["pin_resp"].copy_(b["resp"], non_blocking=True)
        stream.synchronize()
        chi_out = b["pin_chi2"].numpy()[:n_bands].copy()
        chi_derivs = response_view(b["pin_resp"].numpy(), n_bands, n_sources).copy()
        if patch.return_residual:
            residuals = patch.retrieve_array("residual")
            if unpack:
                residuals = self.unpack_residuals(residuals, patch)
            return chi_out, chi_derivs, residuals
        return chi_out, chi_derivs
