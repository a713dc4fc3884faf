"""Patches across GPUs: one process per GPU, each evaluating its own patches.

The reference scales out with an MPI task farm: a parent checks regions out of
the superscene and sends each to a child, which builds the patch, evaluates
and fits it on its own GPU, and sends the result back (forcepho/dispatcher.py:
156-300).  Patches are independent, so the B200 counterpart has no data-path
collective: every rank owns a fixed share of the patches (assigned once,
longest work first, to balance the ranks) and evaluates them with its own
batched plan; results are gathered to one rank only when the caller wants
them there.  ``torch.distributed`` provides the process group (NCCL on GPUs,
gloo on CPUs); the only collectives are ``gather_object`` of per-patch results
and small reductions of timings.

One patch can also be split over ranks by exposure (``SplitPatchProposer``):
chi2 and its gradients are sums over pixels, hence over exposures, so every
rank evaluates the exposures assigned to it as a patch of its own
(``exposure_subpatch``) and one all-reduce of n_bands x (1 + 7 n_sources)
doubles gives every rank the whole patch's result.  That trades one small
collective per evaluation for latency on patches too large for one GPU's
turnaround.
"""

import heapq

import numpy as np

__all__ = ["balance", "local_indices", "gather_results", "PatchFarm", "exposure_weights", "exposure_subpatch",
           "SplitPatchProposer"]


def balance(weights, world):
    """Assign items to ``world`` ranks, largest weight first, each to the rank
    with the least total so far (ties: lowest rank).  Deterministic; returns a
    list of sorted index lists."""
    w = np.asarray(weights, dtype=np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + w[i], r))
    return [sorted(x) for x in out]


def local_indices(weights, rank, world):
    return balance(weights, world)[rank]


def gather_results(local, indices, n_total, dst=0, group=None):
    """Gather per-item results of every rank into global order on ``dst``
    (a list of length n_total there, None on other ranks)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    payload = list(zip(indices, local))
    bucket = [None] * world if rank == dst else None
    dist.gather_object(payload, bucket, dst=dst, group=group)
    if rank != dst:
        return None
    out = [None] * n_total
    for part in bucket:
        for i, r in part:
            out[i] = r
    return out


class PatchFarm:
    """This rank's share of a list of patches and its evaluator.

    Parameters
    ----------
    make_patch : callable(i) -> patch, builds global patch i (called only for
        this rank's indices)
    weights : per-patch work estimates (e.g. pixel-Gaussian pairs)
    rank, world : this process and the number of processes
    evaluator : callable(list of local patches) -> callable(list of proposals)
        -> list of results; defaults to a ``BatchedProposer`` on the current
        CUDA device, so each rank selects its GPU first
        (``torch.cuda.set_device(local_rank)``)
    """

    def __init__(self, make_patch, weights, rank, world, evaluator=None):
        self.rank, self.world = rank, world
        self.n_total = len(weights)
        self.indices = local_indices(weights, rank, world)
        self.patches = [make_patch(i) for i in self.indices]
        if evaluator is None:
            from .batch import BatchedProposer

            def evaluator(patches):
                for p in patches:
                    if getattr(p, "device_patch", None) is None:
                        p.send_to_device()
                bp = BatchedProposer(patches)
                return bp.evaluate_proposals
        self._eval = evaluator(self.patches) if self.patches else (lambda props: [])

    def evaluate(self, proposals_global):
        """Evaluate this rank's patches; ``proposals_global`` maps global index
        to proposal (list or dict).  Returns this rank's results in local order."""
        return self._eval([proposals_global[i] for i in self.indices])

    def evaluate_and_gather(self, proposals_global, dst=0, group=None):
        return gather_results(self.evaluate(proposals_global), self.indices, self.n_total, dst=dst, group=group)


# ---------------------------------------------------------------------------
# one patch over several ranks, split by exposure
# ---------------------------------------------------------------------------
# attributes of a patch that belong to its device copy, not to its arrays
_DEVICE_STATE = ("device_ptrs", "device_patch", "patch_struct", "device_generation", "data_generation")
# per-exposure lists and arrays some patch classes carry besides the kernel's:
# synthetic patches (PSF blocks, stamp shapes, noise levels) and store-backed
# ones (headers, WCS, exposure paths, band names, background offsets)
_PER_EXPOSURE = ("psf_blocks", "original_shapes", "original_sizes", "sigma", "hdrs", "wcses", "epaths", "bands",
                 "background_offsets")


def _band_of_exposure(patch):
    return np.repeat(np.arange(patch.n_bands), np.asarray(patch.band_N, dtype=np.int64))


def exposure_weights(patch):
    """Pixel-Gaussian pairs of every exposure of ``patch``: its pixels times
    n_sources x n_psf_per_source of its band."""
    nb = np.asarray(patch.n_psf_per_source, dtype=np.int64)[_band_of_exposure(patch)]
    return np.asarray(patch.exposure_N, dtype=np.int64) * int(patch.n_sources) * nb


def exposure_subpatch(patch, exposures):
    """A new patch of the same class holding only ``exposures`` (indices into
    the patch's exposures, kept in band order) and every band of ``patch``.
    A band none of whose exposures is kept has ``band_N = 0``: its chi2 and
    gradients are zero.  The kernel's results are sums over exposures, so the
    results of the sub-patches of a partition of the exposures add up to the
    whole patch's.  The sub-patch shares the scene and per-band metadata,
    gets copies of the per-exposure arrays (pixels, astrometry, PSF
    mixtures) and has no device copy until ``send_to_device``."""
    ex = np.array(sorted({int(e) for e in exposures}), dtype=np.int64)
    ne = patch.n_exp
    if len(ex) and (ex[0] < 0 or ex[-1] >= ne):
        raise ValueError("exposure indices must lie in [0, %d)" % ne)
    cls = type(patch)
    sub = cls.__new__(cls)
    sub.__dict__.update({k: v for k, v in patch.__dict__.items() if k not in _DEVICE_STATE})
    band = _band_of_exposure(patch)
    es = np.asarray(patch.exposure_start, dtype=np.int64)
    en = np.asarray(patch.exposure_N, dtype=np.int64)
    for name in ("xpix", "ypix", "data", "ierr"):
        arr = getattr(patch, name)
        parts = [arr[es[e]:es[e] + en[e]] for e in ex]
        setattr(sub, name, np.concatenate(parts) if parts else arr[:0].copy())
    n_new = en[ex]
    sub.exposure_N = n_new.astype(np.asarray(patch.exposure_N).dtype)
    sub.exposure_start = (np.cumsum(n_new) - n_new).astype(np.asarray(patch.exposure_start).dtype)
    bn = np.bincount(band[ex], minlength=patch.n_bands)
    sub.band_N = bn.astype(np.asarray(patch.band_N).dtype)
    sub.band_start = (np.cumsum(bn) - bn).astype(np.asarray(patch.band_start).dtype)
    for name in ("D", "CW", "crpix", "crval", "G"):
        setattr(sub, name, np.ascontiguousarray(np.asarray(getattr(patch, name))[ex]))
    npsf = np.asarray(patch.n_psf_per_source, dtype=np.int64)
    ps = np.asarray(patch.psfgauss_start, dtype=np.int64)
    # each exposure's block: one PSF mixture per source (the kernel reads the
    # first n_psf entries of it)
    blocks = [patch.psfgauss[ps[e]:ps[e] + max(int(patch.n_sources), 1) * npsf[band[e]]] for e in ex]
    sub.psfgauss = np.concatenate(blocks) if blocks else patch.psfgauss[:0].copy()
    lens = np.array([len(b) for b in blocks], dtype=np.int64)
    sub.psfgauss_start = (np.cumsum(lens) - lens).astype(np.asarray(patch.psfgauss_start).dtype)
    for name in _PER_EXPOSURE:
        v = getattr(patch, name, None)
        if v is not None and len(v) == ne:
            setattr(sub, name, [v[e] for e in ex] if isinstance(v, list) else np.asarray(v)[ex])
    if getattr(patch, "n_exp_per_band", None) is not None:
        sub.n_exp_per_band = np.asarray(sub.band_N).astype(np.asarray(patch.n_exp_per_band).dtype)
    ast = getattr(patch, "astrometry", None)
    if isinstance(ast, tuple) and all(len(a) == ne for a in ast):
        sub.astrometry = tuple(np.asarray(a)[ex] for a in ast)
    sub._dirty_data = True
    sub.exposures_of_parent = ex
    return sub


class SplitPatchProposer:
    """One patch evaluated by all ranks of a process group, split by exposure.

    Every rank holds the exposures ``balance`` gives it by pixel-Gaussian
    pairs (``exposures``) as a sub-patch on its own device, evaluates it, and
    one ``all_reduce`` (sum) of n_bands x (1 + 7 n_sources) doubles gives every
    rank the whole patch's ``(chi2 f64[n_bands], chi2_derivs f32[n_bands,
    n_sources, 7])``, the shapes of ``GPUProposer.evaluate_proposal``.  The
    ranks' chi2 (FP64) and FP32 gradients are summed in FP64, and the
    gradient sums rounded to FP32 once more.  With NCCL the reduced
    buffer lives on the current CUDA device; with gloo on the host.  Every
    rank must call ``evaluate_proposal`` with the same proposal, in the same
    order (it is a collective).

    ``proposer`` (default ``B200Proposer``) evaluates the local sub-patch:
    any object with ``evaluate_proposal(proposal, patch=...)`` returning
    (chi2, chi2_derivs).  A rank given no exposures evaluates nothing and
    contributes zeros.
    """

    def __init__(self, patch, rank=0, world=1, group=None, proposer=None, send=True):
        self.rank, self.world, self.group = rank, world, group
        self.n_bands, self.n_sources = patch.n_bands, int(patch.n_sources)
        self.exposures = balance(exposure_weights(patch), world)[rank]
        self.patch = exposure_subpatch(patch, self.exposures) if self.exposures else None
        if self.patch is not None:
            self.patch.return_residual = False
            if send:
                self.patch.send_to_device()
        if proposer is None and self.patch is not None:
            from .proposal import B200Proposer
            proposer = B200Proposer()
        self.proposer = proposer

    def evaluate_local(self, proposal):
        """This rank's part, not reduced: n_bands chi2 terms then the
        n_bands x n_sources x 7 gradient terms, as one FP64 vector (zeros for
        a rank without exposures)."""
        nb, ns = self.n_bands, self.n_sources
        buf = np.zeros(nb * (1 + ns * 7), dtype=np.float64)
        if self.patch is not None:
            chi2, dchi2 = self.proposer.evaluate_proposal(proposal, patch=self.patch)[:2]
            buf[:nb] = chi2
            buf[nb:] = np.asarray(dchi2, dtype=np.float64).reshape(-1)
        return buf

    def unpack(self, buf):
        nb, ns = self.n_bands, self.n_sources
        return buf[:nb].copy(), buf[nb:].reshape(nb, ns, 7).astype(np.float32)

    def evaluate_proposal(self, proposal, **kwargs):
        import torch
        buf = self.evaluate_local(proposal)
        if self.world > 1:
            import torch.distributed as dist
            t = torch.from_numpy(buf)
            if dist.get_backend(self.group) == "nccl":
                t = t.to(torch.device("cuda", torch.cuda.current_device()))
            dist.all_reduce(t, group=self.group)
            buf = t.cpu().numpy()
        return self.unpack(buf)
