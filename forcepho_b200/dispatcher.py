"""Regions of a scene worked in batches, one process per GPU.

The reference's parent process checks regions out of the superscene one at a
time and hands each to an idle MPI child, which builds the patch, samples it
on its GPU and sends the result back to be checked in
(forcepho/dispatcher.py:29-300).  One patch per GPU leaves a B200 mostly idle,
so here the unit of work is a *batch*: every round, rank 0 checks out as many
regions as all ranks take together (``batch_per_rank`` each, while the scene
stays sparse), splits them over the ranks by estimated work (largest first),
every rank works its share in one call -- one batched launch for the whole
share -- and rank 0 checks the results back in, in task order.  Regions
checked out together never share an active source, so the ranks exchange
nothing but the task descriptions and results: Python objects over
``torch.distributed`` (``broadcast_object_list``, ``gather_object``; NCCL or
gloo), never pixels.  The rounds are synchronous, so for a given seed the
scene evolves identically for any number of ranks with the same total batch.

* ``checkout_batch``  -- the parent's checkout loop (``ntry`` draws per region);
* ``run``             -- the round loop on every rank;
* ``dummy_work``      -- the reference's test work unit, without the sleep;
* ``flux_fit_work``   -- a GPU work unit: pack each region's patch from the
  stores, subtract its fixed sources, solve the active sources' fluxes, and
  evaluate chi2 and gradients of all the share's patches in one launch;
* ``hmc_work``        -- a GPU work unit that samples all the share's patches
  together with device-resident HMC, as the reference's child samples one.
"""

import time

import numpy as np

from .distributed import balance

__all__ = ["checkout_batch", "task_weight", "run", "dummy_work", "flux_fit_work", "hmc_work"]


def checkout_batch(scene, n_max, ntry=1000, first_taskid=0):
    """Up to ``n_max`` regions checked out of ``scene``: for each, up to
    ``ntry`` seed draws until one gives a region; stops early when a region
    cannot be found, the scene is no longer sparse or no source is left to
    seed a region.  Returns task dicts
    (taskid, region, active, fixed, bounds, cov, bands, shape_cols)."""
    tasks = []
    while len(tasks) < n_max and scene.sparse:
        w = scene.seed_weight()
        if not (len(w) and np.all(np.isfinite(w)) and w.sum() > 0):
            break                               # every source is checked out
        for _ in range(ntry):
            region, active, fixed = scene.checkout_region()
            if active is not None:
                break
        else:
            break
        bounds, cov = scene.bounds_and_covs(active["source_index"])
        tasks.append(dict(taskid=first_taskid + len(tasks), region=region, active=active, fixed=fixed,
                          bounds=bounds, cov=cov, bands=list(scene.bands), shape_cols=list(scene.shape_cols)))
    return tasks


def task_weight(task):
    """Relative cost of a task: active sources times the region's area."""
    return float(len(task["active"])) * float(task["region"].radius) ** 2


def run(scene, work, batch_per_rank=8, rank=0, world=1, group=None, ntry=1000, max_rounds=None, log=None):
    """Work the scene in rounds until no source needs more iterations (or
    ``max_rounds``).  ``scene`` is the SuperScene on rank 0 (None elsewhere);
    ``work(tasks)`` returns one result dict per task with ``final`` (the
    active rows with new parameters) and optionally ``niter`` (default 1)
    and ``covs``.  Every rank calls this; returns per-round records on rank 0
    (rounds, tasks, seconds) and None elsewhere.  An exception in ``work`` on
    one rank ends that rank's call; the others then fail in the round's
    ``gather_object`` when the process group's timeout runs out, so give the
    group a short timeout."""
    import torch.distributed as dist
    distributed = world > 1
    rounds, taskid = [], 0
    while True:
        t0 = time.perf_counter()
        if rank == 0:
            done = (not scene.undone) or (max_rounds is not None and len(rounds) >= max_rounds)
            tasks = [] if done else checkout_batch(scene, batch_per_rank * world, ntry=ntry, first_taskid=taskid)
            taskid += len(tasks)
            shares = [[tasks[i] for i in idx] for idx in balance([task_weight(t) for t in tasks], world)]
            msg = [None if (done or not tasks) else shares]
        else:
            msg = [None]
        if distributed:
            dist.broadcast_object_list(msg, src=0, group=group)
        if msg[0] is None:
            break
        mine = msg[0][rank]
        results = work(mine) if mine else []
        if len(results) != len(mine):
            raise RuntimeError("work returned %d results for %d tasks" % (len(results), len(mine)))
        for t, r in zip(mine, results):
            r.setdefault("taskid", t["taskid"])
        if distributed:
            gathered = [None] * world if rank == 0 else None
            dist.gather_object(results, gathered, dst=0, group=group)
        else:
            gathered = [results]
        if rank == 0:
            by_id = {t["taskid"]: t for t in tasks}
            for r in sorted((r for part in gathered for r in part), key=lambda r: r["taskid"]):
                t = by_id[r["taskid"]]
                scene.checkin_region(r["final"], t["fixed"], niter=r.get("niter", 1), block_covs=r.get("covs"),
                                     taskID=r["taskid"])
            rec = dict(round=len(rounds), tasks=len(tasks), per_rank=[len(s) for s in msg[0]],
                       seconds=time.perf_counter() - t0)
            rounds.append(rec)
            if log is not None:
                log(rec)
    return rounds if rank == 0 else None


def dummy_work(tasks, niter=75):
    """The reference's stand-in work unit (dispatcher.py:290-304): parameters
    unchanged, ``niter`` iterations counted."""
    return [dict(final=t["active"].copy(), niter=niter) for t in tasks]


def flux_fit_work(make_patcher, allbands, niter=1, tile_pixels=256, keep_patches=False):
    """A GPU work unit over a share of regions.  For each task: pack the
    region's patch (``make_patcher()`` returns an empty store-backed patch),
    subtract the fixed sources' models on the device and solve the active
    sources' fluxes band by band (the linear step of the reference's
    ``run_opt``, fitting.py:590-620).  Then chi2 and its gradients at the new
    fluxes for every patch of the share in one batched launch.  Each result
    carries ``final`` (active rows with the fitted fluxes), ``chi2`` and
    ``dchi2`` (and, with ``keep_patches``, the still-resident ``patch``)."""
    from .batch import BatchedProposer
    from .fitting import optimize_fluxes

    def work(tasks):
        patches, finals = [], []
        for t in tasks:
            p = make_patcher()
            p.build_patch(t["region"], None, allbands=allbands)
            if t["fixed"] is not None and len(t["fixed"]):
                p.subtract_fixed(t["fixed"], active=t["active"], swap_local=True)
            else:
                p.pack_meta(p.set_scene(t["active"]))
                p.send_to_device()
            fit = optimize_fluxes(p, t["active"])
            if not isinstance(fit[0], list):
                raise RuntimeError("flux solve failed for task %d in band %d" % (t["taskid"], fit[0]))
            final = t["active"].copy()
            for b, flux in zip(p.bandlist, fit[0]):
                final[b] = flux
            # the active scene at the fitted fluxes (positions, hence the device
            # metadata, unchanged); the device data stays the fixed-subtracted image
            scene = p.set_scene(final)
            p.zerocoords(scene, sky_zero=p.patch_reference_coordinates)
            p.scene = scene
            patches.append(p)
            finals.append(final)
        bp = BatchedProposer(patches, tile_pixels=tile_pixels, use_graph=False)
        res = bp.evaluate_proposals([p.scene.get_proposal() for p in patches])
        out = [dict(final=f, niter=niter, chi2=c, dchi2=d) for f, (c, d) in zip(finals, res)]
        for r, p in zip(out, patches):
            if keep_patches:
                r["patch"] = p
            else:
                p.free()
        return out

    return work


def _prepared_patch(make_patcher, task, allbands):
    """The task region's patch on the device, fixed sources subtracted, the
    active scene's metadata packed, no residual buffer; and that scene."""
    p = make_patcher()
    p.build_patch(task["region"], None, allbands=allbands)
    if task["fixed"] is not None and len(task["fixed"]):
        _, scene = p.subtract_fixed(task["fixed"], active=task["active"], swap_local=True)
        p.device_ptrs.pop("residual", None)
        p.return_residual = False
        p.send_patchstruct_to_device()
    else:
        scene = p.set_scene(task["active"])
        p.pack_meta(scene)
        p.return_residual = False
        p.send_to_device()
    return p, scene


def hmc_work(make_patcher, allbands, n_warmup=40, n_draws=40, n_steps=16, seed=0, tile_pixels=1024):
    """A GPU sampling work unit over a share of regions: the counterpart of the
    reference child's ``run_lmc`` on one patch (fitting.py:254-341), for all
    the share's patches at once with ``hmc.DeviceHMC``.  Each region's patch is
    packed, its fixed sources subtracted on the device, and its active
    sources sampled within the task's prior bounds: step sizes adapted by
    dual averaging over the first half of the ``n_warmup`` trajectories, the
    diagonal mass matrix then taken from the second half's draws, then
    ``n_draws`` recorded trajectories.  Each result carries ``final`` (the
    active rows at the posterior mean), ``covs`` (per-source covariance of
    the draws when the patch has every scene band), ``niter`` = n_draws, and
    the acceptance rate of every patch."""
    import torch
    from .hmc import DeviceHMC
    from .superscene import bounds_vectors
    if n_draws < 1 or n_warmup < 0 or n_steps < 1:
        raise ValueError("hmc_work needs n_draws >= 1, n_warmup >= 0 and n_steps >= 1")

    def work(tasks):
        patches, scenes, theta0, bounds = [], [], [], []
        for t in tasks:
            p, scene = _prepared_patch(make_patcher, t, allbands)
            lo, hi = bounds_vectors(t["bounds"], p.bandlist, shapenames=t["shape_cols"],
                                    reference_coordinates=p.patch_reference_coordinates)
            patches.append(p)
            scenes.append(scene)
            theta0.append(np.clip(scene.get_all_source_params(), lo, hi))
            bounds.append((lo, hi))
        n1 = n_warmup // 2
        n2 = n_warmup - n1
        h = DeviceHMC(patches, theta0, bounds=bounds, n_steps=n_steps, max_traj=n_warmup + 2 * n_draws + 2,
                      seed=seed, tile_pixels=tile_pixels)
        h.estimate_inv_mass()
        h.run(n1, adapt=True)
        h.end_adaptation()
        f64 = dict(dtype=torch.float64, device=h.device)
        warm = torch.zeros((max(n2, 1), h.n_params), **f64)
        h.run(n2, adapt=True, record={i: warm[i] for i in range(n2)})
        h.end_adaptation()
        if n2 >= 2:
            h.adapt_mass_from(warm[:n2])
        h.start_adaptation()
        h.run(max(n_draws // 2, 1), adapt=True)
        h.end_adaptation()
        acc0 = h.accepted.clone()
        draws = torch.zeros((max(n_draws, 1), h.n_params), **f64)
        h.run(n_draws, record={i: draws[i] for i in range(n_draws)})
        rate = ((h.accepted - acc0).double() / max(n_draws, 1)).cpu().numpy()
        theta = (h.lower + (h.upper - h.lower) * torch.sigmoid(draws[:n_draws])).cpu().numpy()
        out = []
        for i, (t, p) in enumerate(zip(tasks, patches)):
            th = theta[:, h.slices[i]]
            ns = int(p.n_sources)
            npar = p.n_bands + 6
            mean = th.mean(axis=0).reshape(ns, npar)
            final = t["active"].copy()
            ra0, dec0 = p.patch_reference_coordinates
            for j, b in enumerate(p.bandlist):
                final[b] = mean[:, j]
            for j, c in enumerate(t["shape_cols"]):
                final[c] = mean[:, p.n_bands + j]
            final["ra"] += ra0
            final["dec"] += dec0
            covs = None
            if list(p.bandlist) == list(t["bands"]) and n_draws >= 2:
                blocks = th.reshape(n_draws, ns, npar)
                covs = np.stack([np.cov(blocks[:, k, :], rowvar=False) for k in range(ns)])
            out.append(dict(final=final, covs=covs, niter=n_draws, acceptance=float(rate[i])))
        for p in patches:
            p.free()
        return out

    return work
