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
"""

import heapq

import numpy as np

__all__ = ["balance", "local_indices", "gather_results", "PatchFarm"]


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
