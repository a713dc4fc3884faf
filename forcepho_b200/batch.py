"""Many patches, one pass: the batched evaluation of the likelihood hot path.

The reference evaluates one patch per call: ``GPUProposer.evaluate_proposal``
launches ``EvaluateProposal`` with one CTA per band (forcepho/proposal.py:96-152)
and scales out by farming patches to MPI ranks (forcepho/dispatcher.py:156-300).
On a B200 a single patch of a few bands fills a handful of the 148 SMs, so
``BatchedProposer`` evaluates one proposal for each of many device-resident
patches in one pass: a single work plan over all their pixel tiles, one
persistent tile launch, and a fixed-order reduction per (patch, band).  The
three launches of one evaluation are captured once into a CUDA graph and
replayed.

``evaluate_proposals(list of source_struct arrays)`` is the public call:
host proposals -> pinned staging -> device, graph replay, chi2 and Response
records back to the host, returned per patch in the reference's shapes.
"""

import numpy as np
import torch

from . import _native as N
from .autotune import Autotuner, size_class
from .device import Plan, pack_proposals
from .kernel_limits import MAXBANDS, MAXSOURCES, NPARAMS
from .structs import source_struct_dtype

__all__ = ["BatchedProposer", "render_models"]

# a source record as raw bytes, for plain copies into the pinned staging buffer
_RECORD = np.dtype("V%d" % source_struct_dtype.itemsize)
_ZERO_RECORD = np.zeros(1, dtype=source_struct_dtype).view(_RECORD)[0]


class BatchedProposer:
    """One proposal per patch for a list of device patches (``send_to_device``-ed).

    Parameters
    ----------
    patches : list of patches with ``B200PatchMixin``
    tile_pixels, ctas_per_sm : launch parameters; ``autotune=True`` times the
        candidates on the device and keeps the fastest.
    use_graph : capture the evaluation into a CUDA graph on first use.
    """

    def __init__(self, patches, tile_pixels=1024, ctas_per_sm=4, flags=0, autotune=False,
                 use_graph=True, tuner=None, tile_classes=None):
        N.load()
        self.patches = list(patches)
        self.n = len(self.patches)
        self.flags = flags
        self.use_graph = use_graph
        self.graph = None
        self.tune_log = []
        if autotune:
            tuner = tuner or Autotuner()
            self._autotune(tuner, per_class=autotune == "classes")
        else:
            self.plan = Plan(self.patches, tile_pixels=tile_pixels, tile_classes=tile_classes)
            self.launch = self.plan.launch(ctas_per_sm=ctas_per_sm, flags=flags)
        self._init_host_buffers()

    def _init_host_buffers(self):
        """Pinned staging for proposals and compact results.

        Proposals: the device layout, [n_patches][MAXSOURCES] records, written
        patch by patch as raw 264-byte records; a slot left over from a longer
        earlier proposal is zeroed.  Results: only the (patch, band) rows that
        exist are gathered on the device and copied back (chi2 and Response
        records), in patch-major, band-minor order."""
        dev = self.plan.device
        self._pin_prop = torch.zeros(self.plan.proposals.numel(), dtype=torch.uint8).pin_memory()
        self._prop_slots = self._pin_prop.numpy().view(_RECORD).reshape(self.n, MAXSOURCES)
        self._prop_len = [0] * self.n
        nb = [int(p.n_bands) for p in self.patches]
        rows = [i * MAXBANDS + b for i in range(self.n) for b in range(nb[i])]
        self._rows = torch.tensor(rows, dtype=torch.int64, device=dev)
        self._dev_chi2 = torch.zeros(len(rows), dtype=torch.float64, device=dev)
        self._dev_resp = torch.zeros((len(rows), MAXSOURCES * NPARAMS), dtype=torch.float32, device=dev)
        self._pin_chi2 = torch.zeros(len(rows), dtype=torch.float64).pin_memory()
        self._pin_resp = torch.zeros((len(rows), MAXSOURCES * NPARAMS), dtype=torch.float32).pin_memory()
        offsets = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(int)
        self._slices = [(slice(int(o), int(o) + nb[i]), (slice(int(o), int(o) + nb[i]),
                                                         slice(0, int(self.patches[i].n_sources))))
                        for i, o in enumerate(offsets)]
        # completion of the last copy out of the proposal staging buffer and of
        # the last copy into the result buffers: the host waits on them before
        # rewriting the one or reading the others
        self._h2d_done = None
        self._d2h_done = None

    # --- launch parameters ---
    def _autotune(self, tuner, per_class=False):
        """Time the candidates and keep the fastest: one tile size for the
        plan, or (``per_class``) one per exposure-size class."""
        props = self._current_proposals()

        def make_plan(tp=None, classes=None):
            pl = Plan(self.patches, tile_pixels=tp or 1024, tile_classes=classes)
            pl.proposals.copy_(torch.from_numpy(props.view(np.uint8).reshape(-1)))
            return pl

        n_pairs = sum(p.n_pairs() for p in self.patches)
        key = size_class(n_pairs, sum(p.npix for p in self.patches) // 1024)
        if per_class:
            classes, cps, ms = tuner.tune_classes(key, lambda cl: make_plan(classes=cl))
            self.tune_log = [r for r in tuner.log if r[0][1:] == key]
            self.plan = Plan(self.patches, tile_classes=classes)
        else:
            tp, cps, ms = tuner.tune(key, make_plan)
            self.tune_log = [r for r in tuner.log if r[0] == key]
            self.plan = Plan(self.patches, tile_pixels=tp)
        self.launch = self.plan.launch(ctas_per_sm=cps, flags=self.flags)
        self.plan.proposals.copy_(torch.from_numpy(props.view(np.uint8).reshape(-1)))

    @property
    def tile_classes(self):
        """[(max exposure pixels, tile pixels), ...] of the plan (one class when uniform)."""
        return self.plan.tile_classes or [(2 ** 31 - 1, self.plan.tile_pixels)]

    def _current_proposals(self):
        return pack_proposals([p.scene.get_proposal() if getattr(p, "scene", None) is not None
                               else np.zeros(int(p.n_sources), source_struct_dtype) for p in self.patches],
                              self.n)

    @property
    def n_pairs(self):
        return self.plan.n_pairs

    @property
    def tile_pixels(self):
        return self.plan.tile_pixels

    # --- device-side pieces (no host synchronisation) ---
    def set_proposals_async(self, proposals, stream=None):
        """Stage host proposals (list of ``source_struct_dtype`` arrays, one per
        patch; patches past the end of the list get no sources) and queue
        their copy to the device."""
        if len(proposals) > self.n:
            raise ValueError("%d proposals for %d patches" % (len(proposals), self.n))
        s = stream or torch.cuda.current_stream()
        self.plan.check_current(s)           # a captured graph replays the plan's tables
        if self._h2d_done is not None:
            self._h2d_done.synchronize()     # the previous copy may still read the buffer
        slots, lens = self._prop_slots, self._prop_len
        for i in range(self.n):
            if i < len(proposals):
                p = proposals[i]
                if not (type(p) is np.ndarray and p.dtype == source_struct_dtype and p.ndim == 1
                        and p.flags.c_contiguous):
                    p = np.ascontiguousarray(np.asarray(p).astype(source_struct_dtype, copy=False)).reshape(-1)
                k = len(p)
                if k > MAXSOURCES:
                    raise ValueError("proposal %d has %d sources > MAXSOURCES=%d" % (i, k, MAXSOURCES))
                slots[i, :k] = p.view(_RECORD)
            else:
                k = 0
            if k < lens[i]:
                slots[i, k:lens[i]] = _ZERO_RECORD
            lens[i] = k
        with torch.cuda.stream(s):
            self.plan.proposals.copy_(self._pin_prop, non_blocking=True)
        self._h2d_done = torch.cuda.Event()
        self._h2d_done.record(s)

    def run(self, stream=None):
        """Queue one evaluation of the device proposals (graph replay when captured)."""
        s = stream or torch.cuda.current_stream()
        self.plan.check_current(s)           # raises on a stale plan, re-packs swapped data
        if self.use_graph:
            if self.graph is None:
                self.capture(s)
            with torch.cuda.stream(s):
                self.graph.replay()
        else:
            self.plan.evaluate(self.launch, stream=s)

    def capture(self, stream=None):
        s = stream or torch.cuda.current_stream()
        # one eager evaluation first: sets kernel attributes outside capture
        self.plan.evaluate(self.launch, stream=s)
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.plan.evaluate(self.launch)
        torch.cuda.synchronize()
        self.graph = g
        return g

    def fetch_async(self, stream=None):
        """Queue the device gather of the existing (patch, band) rows and their
        copy into pinned host memory."""
        s = stream or torch.cuda.current_stream()
        with torch.cuda.stream(s):
            torch.index_select(self.plan.chi2.view(-1), 0, self._rows, out=self._dev_chi2)
            torch.index_select(self.plan.response.view(-1, MAXSOURCES * NPARAMS), 0, self._rows,
                               out=self._dev_resp)
            self._pin_chi2.copy_(self._dev_chi2, non_blocking=True)
            self._pin_resp.copy_(self._dev_resp, non_blocking=True)
        self._d2h_done = torch.cuda.Event()
        self._d2h_done.record(s)

    def results(self):
        """Per patch (chi2[n_bands] f64, dchi2[n_bands, n_sources, 7] f32) from the
        last fetch (waiting for its copies to land): views into one fresh copy
        of the fetched rows, so they stay valid after later calls."""
        if self._d2h_done is not None:
            self._d2h_done.synchronize()
        c = self._pin_chi2.numpy().copy()
        r = self._pin_resp.numpy().copy().reshape(-1, MAXSOURCES, NPARAMS)
        return [(c[a], r[b]) for a, b in self._slices]

    # --- the public call ---
    def evaluate_proposals(self, proposals, stream=None):
        """Evaluate one proposal (``source_struct_dtype`` array) per patch.

        Returns a list of (chi2, chi2_derivs) per patch with the shapes
        ``GPUProposer.evaluate_proposal`` returns."""
        s = stream or torch.cuda.current_stream()
        self.set_proposals_async(proposals, s)
        self.run(s)
        self.fetch_async(s)
        s.synchronize()
        return self.results()

    # --- transfer accounting of one evaluate_proposals call ---
    @property
    def h2d_bytes(self):
        return int(self.plan.proposals.numel())

    @property
    def d2h_bytes(self):
        return int(self._pin_chi2.numel() * 8 + self._pin_resp.numel() * 4)

    def count_pairs(self, stream=None):
        """(evaluated pairs, pairs within the cutoff, within-cutoff pairs culled) of one evaluation."""
        import ctypes
        s = stream or torch.cuda.current_stream()
        self.plan.evaluate(self.launch, stream=s)
        counts = torch.zeros(3, dtype=torch.int64, device=self.plan.device)
        pl = self.plan
        N.check(pl.L.fp_count_pairs(pl.d_patches.data_ptr(), ctypes.byref(pl.sizes), ctypes.byref(pl.tables),
                                    pl.workspace.data_ptr(), pl.workspace.numel(), counts.data_ptr(),
                                    ctypes.c_void_p(s.cuda_stream)), "fp_count_pairs")
        s.synchronize()
        return tuple(int(v) for v in counts.cpu())


def render_models(patches, proposals=None, tile_pixels=1024):
    """Model counts of every pixel of every (device) patch at ``proposals``
    (default: each patch's scene), rendered by the tiled kernel as minus the
    residual of an all-zero data array.  Returns a list of f32 host arrays."""
    saved = []
    for p in patches:
        saved.append((p.data, p.return_residual))
        p.data = np.zeros_like(p.data)
        p.return_residual = True
        p.send_to_device()
    bp = BatchedProposer(patches, tile_pixels=tile_pixels, use_graph=False)
    props = proposals or [p.scene.get_proposal() for p in patches]
    bp.evaluate_proposals(props)
    models = [-p.retrieve_array("residual") for p in patches]
    for p, (d, rr) in zip(patches, saved):
        p.data = d
        p.return_residual = rr
        p.free()
    return models


_ = (MAXBANDS, MAXSOURCES, NPARAMS)
