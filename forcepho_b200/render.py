"""Renders, fixed-source subtraction and the linear flux design matrix.

The reference drives these through the same likelihood kernel, one full
evaluation at a time (forcepho/patches/device_patch.py:113-254):

* ``subtract_fixed`` evaluates blocks of at most ``maxactive`` fixed (and "big")
  sources in turn and swaps the device data and residual buffers after each,
  so the device data ends as data minus every fixed model, with the active
  scene's metadata packed (:113-183);
* ``design_matrix`` renders each active source alone (one evaluation per
  source, the residual copied back each time) and divides its model by its
  catalog flux in each band (:185-237);
* ``render`` is meant to return a scene's model images (it fails upstream with
  a NameError, :248).

The B200 versions run the tile kernel with ``FLAG_FORWARD_ONLY`` (model,
residual and chi2 only; the gradient pass, two thirds of the work, is
skipped).  ``design_models`` renders every active source in ONE batched
launch: each source becomes a ``SceneView``, a patch of its own for the work
planner that shares the parent's pixel and index arrays, carries only that
source's metadata, reads an all-zero data array and writes its residual
(minus its model) into its own row of a device matrix.  The flux normal
equations are then formed on the device in FP64 (``normal_equations``), so
the design matrix never has to cross PCIe.

A patch provides ``set_scene(catalog)`` and ``meta_for(scene)`` /
``pack_meta(scene)`` (the reference's store-backed patches do;
``synthetic.SyntheticPatch`` does for the synthetic workloads).
"""

import copy

import numpy as np
import torch

from . import _native as N
from .device import Plan, pack_proposals, to_device_bytes
from .structs import patch_struct_dtype, ptr_dtype, source_struct_dtype

__all__ = ["SceneView", "subtract_fixed", "design_models", "design_matrix", "normal_equations", "render"]

_VIEW_META = ("D", "CW", "crpix", "crval", "psfgauss", "psfgauss_start")


class SceneView:
    """A set of sources over a device patch's pixels, as a patch of its own.

    The device struct points at the parent's pixel, index and PSF-count arrays
    and at this view's own copies of the scene's source metadata; ``data`` and
    ``residual`` are device addresses chosen by the caller (e.g. an all-zero
    array and an output row, so the residual is minus the scene's model)."""

    def __init__(self, parent, scene, data_ptr, residual_ptr):
        if getattr(parent, "device_patch", None) is None:
            raise ValueError("the parent patch must be sent to the device first")
        self.parent = parent
        for name in ("exposure_start", "exposure_N", "band_start", "band_N", "n_psf_per_source",
                     "xpix", "ypix"):
            setattr(self, name, getattr(parent, name))
        meta = parent.meta_for(scene)
        self.n_sources = int(meta["n_sources"])
        dev = parent._dev()
        self._keep = {k: to_device_bytes(np.ascontiguousarray(meta[k]), dev) for k in _VIEW_META}
        s = np.zeros(1, dtype=patch_struct_dtype)
        for name in patch_struct_dtype.names:
            if patch_struct_dtype[name] == ptr_dtype:
                if name in self._keep:
                    s[name] = int(self._keep[name].data_ptr())
                elif name in parent.device_ptrs:
                    s[name] = parent.device_ptrs[name].ptr
            else:
                s[name] = getattr(parent, name)
        s["n_sources"] = self.n_sources
        s["data"] = int(data_ptr)
        s["residual"] = int(residual_ptr)
        self.device_patch = torch.empty(patch_struct_dtype.itemsize, dtype=torch.uint8, device=dev)
        self.device_patch.copy_(torch.from_numpy(s.view(np.uint8).copy()))

    @property
    def npix(self):
        return int(self.xpix.shape[0])

    @property
    def n_bands(self):
        return int(len(self.band_N))

    @property
    def n_exp(self):
        return int(len(self.exposure_N))

    @property
    def device_patch_ptr(self):
        return int(self.device_patch.data_ptr())


def _tile_pixels(patch):
    from .autotune import default_tile_pixels
    return default_tile_pixels(patch)


def _forward_only(views, proposals, ctas_per_sm=4):
    """Queue one forward-only evaluation of the views (one proposal each) on
    the current stream, where every temporary of this module is allocated:
    the caching allocator hands their memory to later work on the same stream
    only, so it can be released while the kernel still runs."""
    plan = Plan(views, tile_pixels=_tile_pixels(views[0]))
    host = pack_proposals(proposals, len(views))
    plan.proposals.copy_(torch.from_numpy(host.view(np.uint8).reshape(-1)))
    plan.evaluate(plan.launch(ctas_per_sm=ctas_per_sm, flags=N.FLAG_FORWARD_ONLY))
    return plan


def _scene_view(patch, scene, data_ptr, residual_ptr):
    """A SceneView of ``scene`` (from ``patch.set_scene``) and the scene, with
    its positions as the offsets the metadata and proposals take.  A
    store-backed patch's ``set_scene`` gives absolute positions (its
    ``pack_meta`` zeroes them): the scene is zeroed at its own median, as the
    reference's ``pack_meta`` does for every scene it renders, and the patch's
    own reference coordinate is left as it was.  A synthetic patch's catalog
    already holds offsets."""
    if not hasattr(patch, "zerocoords"):
        return SceneView(patch, scene, data_ptr, residual_ptr), scene
    saved = np.array(patch.patch_reference_coordinates, dtype=np.float64, copy=True)
    try:
        patch.zerocoords(scene)
        view = SceneView(patch, scene, data_ptr, residual_ptr)
    finally:
        patch.patch_reference_coordinates = saved
    return view, scene


def _scene_proposal(scene):
    srcs = list(scene.sources)
    if not srcs:
        return np.zeros(0, dtype=source_struct_dtype)
    return np.concatenate([s.proposal().copy() for s in srcs])


def _blocks(catalog, maxactive):
    if catalog is None or len(catalog) == 0:
        return []
    return np.array_split(catalog, np.arange(maxactive, len(catalog), maxactive))


def subtract_fixed(patch, fixed, active=None, big=None, maxactive=15, swap_local=False,
                   big_scene_kwargs=None, **scene_kwargs):
    """Subtract the models of ``big`` and ``fixed`` sources from the device data.

    The device data ends as data minus every fixed and big source model; the
    patch's metadata is the ``active`` scene's, ready for proposals.  Blocks of
    at most ``maxactive`` sources are evaluated in turn (big first), each in
    FP32 on the result of the previous one, as the reference does.  Without
    ``active`` the metadata would describe an already subtracted scene, which
    must be asked for with ``swap_local=True``; ``swap_local`` also copies the
    subtracted data into the host ``patch.data``.

    Returns (proposer for the active scene, that scene)."""
    from .proposal import B200Proposer
    scenes = [patch.set_scene(b, **(big_scene_kwargs or {})) for b in _blocks(big, maxactive)]
    scenes += [patch.set_scene(b, **scene_kwargs) for b in _blocks(fixed, maxactive)]
    if active is not None:
        scenes.append(patch.set_scene(active, **scene_kwargs))
    else:
        if not swap_local:
            raise ValueError("no active sources: the metadata would describe an already subtracted "
                             "scene; pass swap_local=True to accept that")
        if not scenes:
            raise ValueError("no scenes to prepare")
        scenes.append(scenes[-1])
    proposer = patch.get_proposer()
    sub = B200Proposer(flags=N.FLAG_FORWARD_ONLY)
    patch.return_residual = True
    patch.pack_meta(scenes[0])
    patch.send_to_device()
    for i, scene in enumerate(scenes[1:]):
        sub.evaluate_proposal(_scene_proposal(scenes[i]), patch=patch)
        patch.pack_meta(scene)
        patch.swap_on_device()
    if swap_local:
        patch.data = patch.retrieve_array("data").copy()
    return proposer, scenes[-1]


def design_models(patch, active):
    """Device matrix f32[n_active, npix]: each active source's model, divided
    by its catalog flux in each band (one batched forward-only launch)."""
    scene = patch.set_scene(active)
    n = len(scene.sources)
    dev = patch._dev()
    X = torch.empty((n, max(patch.npix, 1)), dtype=torch.float32, device=dev)
    if n == 0:
        return X[:, :patch.npix], scene
    zeros = torch.zeros(max(patch.npix, 1), dtype=torch.float32, device=dev)
    from .sources import Scene
    views, props = [], []
    for i, g in enumerate(scene.sources):
        v, one = _scene_view(patch, Scene([copy.copy(g)]), zeros.data_ptr(), X[i].data_ptr())
        views.append(v)
        props.append(_scene_proposal(one))
    plan = _forward_only(views, props)
    X.neg_()                                             # residual of zero data = -model
    flux = torch.tensor(np.array([g.flux for g in scene.sources], dtype=np.float64),
                        dtype=torch.float32, device=dev)
    bounds = np.concatenate([[0], np.cumsum(patch.band_N_pix)]).astype(int)
    for b in range(patch.n_bands):
        X[:, bounds[b]:bounds[b + 1]].div_(flux[:, b:b + 1])
    del plan, views                                      # stream order keeps their memory until done
    return X[:, :patch.npix], scene


def design_matrix(patch, active, proposer=None, **scene_kwargs):
    """The reference's ``design_matrix`` (device_patch.py:185-237): per band the
    f64 matrix X[n_active, n_pix_band] of flux-normalised source models, and the
    device data (after any fixed-source subtraction) split by band.  Assumes
    ``subtract_fixed`` ran when fixed sources are to be excluded."""
    y = patch.retrieve_array("data")
    ys = np.split(y, np.cumsum(patch.band_N_pix[:-1]))
    X, _ = design_models(patch, active)
    Xh = X.cpu().numpy().astype(np.float64)
    Xes = np.split(Xh, np.cumsum(patch.band_N_pix[:-1]), axis=1)
    return Xes, ys


def normal_equations(patch, active):
    """Per band (X_w X_wᵀ, X_w y_w) in FP64 on the device, with X_w = X·ierr and
    y_w = data·ierr over the band's pixels: the flux normal equations of the
    reference's ``optimize_one_band`` (forcepho/fitting.py:572-587) without
    moving the design matrix to the host."""
    X, _ = design_models(patch, active)
    npix = patch.npix
    d = patch.device_ptrs
    y = d["data"].tensor[:npix * 4].view(torch.float32)
    w = d["ierr"].tensor[:npix * 4].view(torch.float32)
    bounds = np.concatenate([[0], np.cumsum(patch.band_N_pix)]).astype(int)
    out = []
    for b in range(patch.n_bands):
        lo, hi = bounds[b], bounds[b + 1]
        wb = w[lo:hi].double()
        Xp = X[:, lo:hi].double() * wb
        yp = y[lo:hi].double() * wb
        out.append((Xp @ Xp.T, Xp @ yp))
    return [(a.cpu().numpy(), v.cpu().numpy()) for a, v in out]


def render(patch, catalog, splinedata=None, unpack=True):
    """Model images of a catalog's sources over the patch's pixels: per
    exposure (``unpack``) or flat, f32, padding included.  The patch's own data
    and metadata are untouched."""
    scene = patch.set_scene(catalog, splinedata=splinedata)
    dev = patch._dev()
    npix = max(patch.npix, 1)
    zeros = torch.zeros(npix, dtype=torch.float32, device=dev)
    out = torch.empty(npix, dtype=torch.float32, device=dev)
    view, scene = _scene_view(patch, scene, zeros.data_ptr(), out.data_ptr())
    plan = _forward_only([view], [_scene_proposal(scene)])
    del plan, view
    model = (-out[:patch.npix]).cpu().numpy()
    if unpack:
        return np.split(model, np.cumsum(patch.exposure_N[:-1]))
    return model
