"""Device residency of patches and the device-resident work plan.

``B200PatchMixin`` is the B200 counterpart of the reference's ``GPUPatchMixin``
(forcepho/patches/device_patch.py:257-390): the same methods with the same
semantics, with torch CUDA tensors owning the device memory instead of pycuda
allocations:

* ``send_to_device``      -- every pixel and metadata array to the device, a
                             residual buffer iff ``return_residual``, then the
                             152-byte Patch struct (device_patch.py:265-297);
* ``replace_device_meta_ptrs`` -- re-send the metadata arrays (:299-308);
* ``send_patchstruct_to_device`` -- rebuild the struct from the current
                             device pointers (:310-341);
* ``swap_on_device``      -- new metadata, swap the data and residual buffers,
                             re-send the struct, so the device "data" becomes
                             the residual of the last evaluation (:343-364);
* ``retrieve_array``      -- copy one pixel array back (:366-372);
* ``free``                -- release everything (:374-390).

Differences, all on the safe side: the struct lives in one persistent device
buffer that is rewritten in stream order (its address never changes, so a
captured CUDA graph or a plan stays valid across swaps); host-side validation
(``PatchBase.validate``) runs before anything is sent.

``Plan`` wraps the C planner: the tile/exposure/band tables of one or many
device patches, their bounding boxes, the workspace and the output buffers.
"""

import ctypes
import itertools

import numpy as np
import torch

from . import _native as N
from .kernel_limits import MAXBANDS, MAXSOURCES, NPARAMS
from .structs import patch_struct_dtype, ptr_dtype, source_struct_dtype, response_struct_dtype

__all__ = ["B200PatchMixin", "Plan", "to_device_bytes", "current_stream_ptr"]


def current_stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def to_device_bytes(arr, device):
    """Copy a numpy array to a new device uint8 tensor (256-byte aligned by torch)."""
    a = np.ascontiguousarray(arr)
    t = torch.empty(max(a.nbytes, 1), dtype=torch.uint8, device=device)
    if a.nbytes:
        t[:a.nbytes].copy_(torch.from_numpy(a.reshape(-1).view(np.uint8)))
    return t


def _ptr(t):
    return int(t.data_ptr())


# numbers each upload of a patch (``send_to_device``): a re-sent patch may get
# the same device addresses back from the allocator with other pixels in them
_UPLOADS = itertools.count(1)


class _DeviceArray:
    """A device copy of a host array: the uint8 tensor plus dtype/shape to read it back."""

    __slots__ = ("tensor", "dtype", "shape")

    def __init__(self, tensor, dtype, shape):
        self.tensor, self.dtype, self.shape = tensor, np.dtype(dtype), tuple(shape)

    @property
    def ptr(self):
        return _ptr(self.tensor)

    def to_host(self):
        n = int(np.prod(self.shape)) * self.dtype.itemsize
        raw = self.tensor[:n].cpu().numpy()
        return raw.view(self.dtype).reshape(self.shape).copy()


class B200PatchMixin:
    """Mix into a ``PatchBase`` subclass to hold the patch on a CUDA device."""

    device = "cuda"

    def get_proposer(self):
        from .proposal import B200Proposer
        return B200Proposer()

    # --- helpers ---
    def _dev(self):
        return torch.device(self.device)

    def _send(self, name):
        arr = np.ascontiguousarray(getattr(self, name))
        return _DeviceArray(to_device_bytes(arr, self._dev()), arr.dtype, arr.shape)

    # --- the GPUPatchMixin surface ---
    def send_to_device(self):
        self.validate()
        self.device_ptrs = {}
        for name in patch_struct_dtype.names:
            if patch_struct_dtype[name] != ptr_dtype or name == "residual":
                continue
            self.device_ptrs[name] = self._send(name)
        if self.return_residual:
            self._alloc_residual()
        self.send_patchstruct_to_device()
        self._dirty_data = False
        self.device_generation = next(_UPLOADS)
        self.data_generation = next(_UPLOADS)
        return self.device_patch

    def _alloc_residual(self):
        t = torch.zeros(max(self.npix, 1) * 4, dtype=torch.uint8, device=self._dev())
        self.device_ptrs["residual"] = _DeviceArray(t, self.pix_dtype, (self.npix,))

    def replace_device_meta_ptrs(self):
        for name in self.meta_names:
            if patch_struct_dtype[name] == ptr_dtype:
                self.device_ptrs[name] = self._send(name)

    def send_patchstruct_to_device(self):
        s = np.zeros(1, dtype=patch_struct_dtype)
        for name in patch_struct_dtype.names:
            if patch_struct_dtype[name] == ptr_dtype:
                if name in self.device_ptrs:
                    s[name] = self.device_ptrs[name].ptr
            else:
                s[name] = getattr(self, name)
        self.patch_struct = s[0]
        host = torch.from_numpy(s.view(np.uint8).copy())
        if getattr(self, "device_patch", None) is None:
            self.device_patch = torch.empty(patch_struct_dtype.itemsize, dtype=torch.uint8, device=self._dev())
        # stream-ordered overwrite: kernels queued earlier still see the old struct
        self.device_patch.copy_(host, non_blocking=False)
        return self.device_patch

    def swap_on_device(self):
        if "residual" not in getattr(self, "device_ptrs", {}):
            raise AssertionError("Must instantiate the Patch with `return_residual=True`")
        self.validate()
        self.replace_device_meta_ptrs()
        d = self.device_ptrs
        d["data"], d["residual"] = d["residual"], d["data"]
        self.send_patchstruct_to_device()
        self._dirty_data = True
        self.data_generation = next(_UPLOADS)     # plans re-pack their pixel records
        return self.device_patch

    def retrieve_array(self, arrname="residual"):
        torch.cuda.current_stream().synchronize()
        return self.device_ptrs[arrname].to_host().astype(self.pix_dtype, copy=False)

    def free(self):
        self.device_ptrs = {}
        self.device_patch = None
        self.device_generation = None

    # --- consumers of the kernel (device_patch.py:113-254), in forcepho_b200.render ---
    def subtract_fixed(self, fixed, active=None, big=None, maxactive=15, swap_local=False,
                       big_scene_kwargs=None, **scene_kwargs):
        from .render import subtract_fixed
        return subtract_fixed(self, fixed, active=active, big=big, maxactive=maxactive,
                              swap_local=swap_local, big_scene_kwargs=big_scene_kwargs, **scene_kwargs)

    def design_matrix(self, active=None, proposer=None, **scene_kwargs):
        from .render import design_matrix
        return design_matrix(self, active, proposer=proposer, **scene_kwargs)

    def render(self, catalog, splinedata=None):
        from .render import render
        return render(self, catalog, splinedata=splinedata)

    # --- extras of this implementation ---
    @property
    def device_patch_ptr(self):
        return _ptr(self.device_patch)

    def plan_signature(self):
        """What a work plan depends on: the upload, the pixel layout and the
        scene's shape."""
        d = self.device_ptrs
        return (getattr(self, "device_generation", None), int(self.n_sources), self.npix, d["xpix"].ptr,
                d["ypix"].ptr,
                tuple(np.asarray(self.exposure_start).tolist()), tuple(np.asarray(self.exposure_N).tolist()),
                tuple(np.asarray(self.band_N).tolist()), tuple(np.asarray(self.n_psf_per_source).tolist()))


class Plan:
    """Device-resident plan of one or many device patches (see ``fp_plan_*``).

    Owns: the device tables, the workspace, the proposal staging buffers and
    the output buffers ``chi2`` f64[n_patches, MAXBANDS] and ``response``
    f32[n_patches, MAXBANDS, MAXSOURCES*NPARAMS]."""

    def __init__(self, patches, tile_pixels=1024, device=None, stream=None, compact_tiles=True, tile_classes=None):
        self.L = N.load()
        self.patches = list(patches)
        self.n = len(self.patches)
        # one tile size for every exposure, or per exposure-size class:
        # tile_classes = [(max_exposure_pixels, tile_pixels), ...] (the last takes the rest)
        self.tile_classes = None if tile_classes is None else [(int(a), int(b)) for a, b in tile_classes]
        rule = N.tile_rule(self.tile_classes or [(2 ** 31 - 1, int(tile_pixels))])
        self.rule = rule
        self.tile_pixels = max(rule.tile_pixels[c] for c in range(rule.n_classes))
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        shapes = [N.patch_shape(p, coordinates=compact_tiles) for p in self.patches]
        self._shapes = (N.PatchShape * self.n)(*shapes)
        self._shape_keep = shapes
        sz = N.PlanSizes()
        N.check(self.L.fp_plan_count_rule(ctypes.addressof(self._shapes), self.n, ctypes.byref(rule),
                                          ctypes.byref(sz)), "fp_plan_count_rule")
        self.sizes = sz
        h_expos = np.zeros(sz.n_exposures, dtype=N.exposure_desc_dtype)
        h_tiles = np.zeros(sz.n_tiles, dtype=N.tile_dtype)
        h_bands = np.zeros(sz.n_band_outputs, dtype=N.band_desc_dtype)
        h_order = np.zeros(sz.n_tiles, dtype=np.int32)
        h_perm = np.zeros(sz.n_perm, dtype=np.int32)
        N.check(self.L.fp_plan_fill_rule(ctypes.addressof(self._shapes), self.n, ctypes.byref(rule),
                                         h_expos.ctypes.data, h_tiles.ctypes.data, h_bands.ctypes.data,
                                         h_order.ctypes.data, h_perm.ctypes.data), "fp_plan_fill_rule")
        self.h_expos, self.h_tiles, self.h_bands, self.h_order = h_expos, h_tiles, h_bands, h_order
        self.h_perm = h_perm
        self.d_expos = to_device_bytes(h_expos, dev)
        self.d_tiles = to_device_bytes(h_tiles, dev)
        self.d_bands = to_device_bytes(h_bands, dev)
        self.d_order = to_device_bytes(h_order, dev)
        self.d_perm = to_device_bytes(h_perm, dev)
        # (x, y, data, ierr) records of every tile pixel in plan order, read by
        # the tile kernel as one 16-byte load per pixel (fp_plan_pack)
        self.d_pix = torch.empty(max(int(sz.n_perm), 1) * 16, dtype=torch.uint8, device=dev)
        self.tables = N.PlanTables(_ptr(self.d_expos), _ptr(self.d_tiles), _ptr(self.d_order),
                                   _ptr(self.d_bands), _ptr(self.d_perm), _ptr(self.d_pix))
        self.d_patches = torch.zeros(self.n, dtype=torch.int64, device=dev)
        # what the tables were made from: each patch's upload and device struct
        # (holding the struct keeps its memory from being reused)
        self._stamps = [(getattr(p, "device_generation", None), p.device_patch) for p in self.patches]
        self.refresh_patch_pointers()
        self._packed = None
        self.pack(stream)
        self.workspace = torch.zeros(max(sz.workspace_bytes, 256), dtype=torch.uint8, device=dev)
        self.proposals = torch.zeros(self.n * MAXSOURCES * source_struct_dtype.itemsize, dtype=torch.uint8,
                                     device=dev)
        self.chi2 = torch.zeros((self.n, MAXBANDS), dtype=torch.float64, device=dev)
        self.response = torch.zeros((self.n, MAXBANDS, MAXSOURCES * NPARAMS), dtype=torch.float32, device=dev)

    def _data_stamps(self):
        return [getattr(p, "data_generation", None) for p in self.patches]

    def pack(self, stream=None):
        """Queue the gather of every tile pixel's (x, y, data, ierr) into the
        plan's records (and the tile boxes) from the patches' current arrays."""
        N.check(self.L.fp_plan_pack(_ptr(self.d_patches), ctypes.byref(self.sizes), ctypes.byref(self.tables),
                                    _ptr(self.d_pix), current_stream_ptr(stream)), "fp_plan_pack")
        self._packed = self._data_stamps()

    def check_current(self, stream=None):
        """Raise if a patch was freed or sent to the device again since the plan
        was made: its tiles, pixel order and boxes describe the old upload.
        Re-pack the pixel records (queued on ``stream``) if a patch's device
        data changed since the last pack (``swap_on_device``).  Every
        evaluation and graph replay of the plan is preceded by this call."""
        for i, (p, (gen, struct)) in enumerate(zip(self.patches, self._stamps)):
            if getattr(p, "device_generation", None) != gen or getattr(p, "device_patch", None) is not struct:
                raise RuntimeError("patch %d was freed or sent to the device again after this plan was made; "
                                   "make a new plan (or proposer) for it" % i)
        if self._data_stamps() != self._packed:
            self.pack(stream)

    def refresh_patch_pointers(self):
        ptrs = torch.tensor([p.device_patch_ptr for p in self.patches], dtype=torch.int64)
        self.d_patches.copy_(ptrs)

    @property
    def n_pairs(self):
        return int(self.sizes.n_pairs)

    def tile_bboxes(self):
        """Host copy of the device-computed tile boxes (xmin, xmax, ymin, ymax)."""
        raw = self.d_tiles[:self.h_tiles.nbytes].cpu().numpy().view(N.tile_dtype)
        return raw["bbox"].copy()

    def launch(self, tile_pixels=None, ctas_per_sm=3, flags=0):
        lp = N.Launch(self.tile_pixels if tile_pixels is None else int(tile_pixels), int(ctas_per_sm),
                      int(flags), 0)
        if lp.tile_pixels != self.tile_pixels:
            raise ValueError("launch tile size %d differs from the plan's %d" % (lp.tile_pixels, self.tile_pixels))
        return lp

    def evaluate(self, launch=None, stream=None, proposals=None, chi2=None, response=None):
        """Queue one evaluation of the proposals in ``self.proposals`` (or the
        given device buffer) on ``stream``; outputs land in ``self.chi2`` /
        ``self.response`` (or the given buffers).  No host synchronisation."""
        self.check_current(stream)
        lp = launch if launch is not None else self.launch()
        props = self.proposals if proposals is None else proposals
        c2 = self.chi2 if chi2 is None else chi2
        rs = self.response if response is None else response
        N.check(self.L.fp_evaluate_batch(
            _ptr(self.d_patches), self.n, ctypes.byref(self.sizes), ctypes.byref(self.tables), _ptr(props),
            _ptr(c2), _ptr(rs), _ptr(self.workspace), self.workspace.numel(), ctypes.byref(lp),
            current_stream_ptr(stream)), "fp_evaluate_batch")

    def read_status(self, stream=None):
        st = ctypes.c_int32(0)
        N.check(self.L.fp_read_status(_ptr(self.workspace), ctypes.byref(st), current_stream_ptr(stream)),
                "fp_read_status")
        return int(st.value)


def pack_proposals(proposals, n_patches):
    """[n_patches][MAXSOURCES] source records (host numpy) from a list of proposal arrays."""
    out = np.zeros((n_patches, MAXSOURCES), dtype=source_struct_dtype)
    for i, p in enumerate(proposals):
        p = np.asarray(p, dtype=source_struct_dtype).reshape(-1)
        if len(p) > MAXSOURCES:
            raise ValueError("proposal %d has %d sources > MAXSOURCES=%d" % (i, len(p), MAXSOURCES))
        out[i, :len(p)] = p
    return out


def response_view(resp_host, n_bands, n_sources):
    """(n_bands, n_sources, NPARAMS) float32 view of Response records, as the
    reference reshapes them (forcepho/proposal.py:139-141)."""
    r = np.asarray(resp_host).reshape(-1, MAXSOURCES, NPARAMS)
    return r[:n_bands, :n_sources]


_ = response_struct_dtype
