"""ctypes binding of the C ABI in ``include/forcepho_b200.h``.

The CUDA library is the only compute path: if it is missing and cannot be
built, importing the device modules raises instead of falling back to
anything else.
"""

import ctypes
import os

import numpy as np

from . import build as _build
from .structs import STRUCT_SIZES

c_i32, c_i64, c_vp, c_sz = ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p, ctypes.c_size_t


class PatchShape(ctypes.Structure):
    _fields_ = [("n_bands", c_i32), ("n_exposures", c_i32), ("n_sources", c_i32), ("n_pix", c_i32),
                ("exposure_start", c_vp), ("exposure_N", c_vp), ("band_start", c_vp),
                ("band_N", c_vp), ("n_psf_per_source", c_vp), ("xpix", c_vp), ("ypix", c_vp)]


class PlanSizes(ctypes.Structure):
    _fields_ = [("n_exposures", c_i64), ("n_tiles", c_i64), ("n_band_outputs", c_i64),
                ("n_gauss", c_i64), ("n_pairs", c_i64), ("n_partials", c_i64),
                ("max_gauss", c_i64), ("workspace_bytes", c_i64), ("n_perm", c_i64)]


class PlanTables(ctypes.Structure):
    _fields_ = [("expos", c_vp), ("tiles", c_vp), ("order", c_vp), ("bands", c_vp), ("perm", c_vp),
                ("pix", c_vp)]


class TileRule(ctypes.Structure):
    _fields_ = [("n_classes", c_i32), ("max_exposure_pixels", c_i32 * 4), ("tile_pixels", c_i32 * 4)]


def tile_rule(classes):
    """TileRule from [(max_exposure_pixels, tile_pixels), ...] (ascending; the
    last class's bound is ignored: it takes every larger exposure)."""
    classes = list(classes)
    if not 1 <= len(classes) <= 4:
        raise ValueError("1 to 4 tile classes")
    r = TileRule()
    r.n_classes = len(classes)
    for c, (mx, tp) in enumerate(classes):
        r.max_exposure_pixels[c] = int(min(mx, 2 ** 31 - 1))
        r.tile_pixels[c] = int(tp)
    return r


class Launch(ctypes.Structure):
    _fields_ = [("tile_pixels", c_i32), ("ctas_per_sm", c_i32), ("flags", c_i32), ("phases", c_i32)]


class SplineTable(ctypes.Structure):
    _fields_ = [("n_radii", c_i32), ("nx", c_i32), ("ny", c_i32), ("kx", c_i32), ("ky", c_i32), ("pad", c_i32),
                ("tx", c_vp), ("ty", c_vp), ("coef", c_vp)]


class HMCState(ctypes.Structure):
    _fields_ = [("n_params", c_i64), ("z", c_vp), ("p", c_vp), ("grad", c_vp), ("z0", c_vp), ("grad0", c_vp),
                ("inv_mass", c_vp), ("eps", c_vp), ("lnp", c_vp), ("lnp0", c_vp), ("h0", c_vp),
                ("energy_error", c_vp), ("accepted", c_vp), ("normals", c_vp), ("uniforms", c_vp),
                ("traj", c_vp), ("n_traj", c_i64)]


HMC_BEGIN, HMC_STEP, HMC_END = 0, 1, 2
NOALLOC_WORKSPACE_BYTES = 32 << 20
hmc_patch_dtype = np.dtype([("param_offset", np.int64), ("n_sources", np.int32), ("n_bands", np.int32)])

FLAG_NO_CULL = 1
FLAG_STATIC = 2
FLAG_FORWARD_ONLY = 4
PHASE_SETUP, PHASE_TILES, PHASE_REDUCE = 1, 2, 4

# device status word bits (include/forcepho_b200.h)
STATUS_TILE_SIZE, STATUS_GAUSS_COUNT, STATUS_SOURCES = 1, 2, 4

# return codes (include/forcepho_b200.h)
FP_OK, FP_ERR_ARGUMENT, FP_ERR_LIMITS, FP_ERR_CUDA, FP_ERR_WORKSPACE, FP_ERR_DEVICE = 0, -1, -2, -3, -4, -5

# numpy mirrors of the plan tables (filled on the host, copied to the device)
exposure_desc_dtype = np.dtype([("gauss_offset", np.int64), ("patch", np.int32), ("exposure", np.int32),
                                ("band", np.int32), ("n_gauss", np.int32), ("n_psf", np.int32),
                                ("n_sources", np.int32)])
tile_dtype = np.dtype([("partial_offset", np.int64), ("expo", np.int32), ("perm_start", np.int32),
                       ("n_pix", np.int32), ("tile_pixels", np.int32), ("bbox", np.float32, 4)])
band_desc_dtype = np.dtype([("patch", np.int32), ("band", np.int32), ("tile_begin", np.int32),
                            ("tile_end", np.int32), ("n_sources", np.int32), ("pad", np.int32)])
assert exposure_desc_dtype.itemsize == 32 and tile_dtype.itemsize == 40 and band_desc_dtype.itemsize == 24

# every entry point of include/forcepho_b200.h with its ctypes signature
SIGNATURES = {
    "fp_error_string": (ctypes.c_char_p, []),
    "fp_version": (ctypes.c_int, []),
    "fp_struct_sizes": (ctypes.c_int, [c_vp]),
    "fp_evaluate_proposal_plain": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, ctypes.c_int, c_vp, c_vp, c_vp]),
    "fp_evaluate_proposal": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, ctypes.c_int, c_vp, c_vp, c_vp]),
    "fp_f64_workspace_bytes": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(c_sz)]),
    "fp_evaluate_proposal_f64": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_vp, c_vp,
                                                c_vp, c_sz, c_vp]),
    "fp_evaluate_proposal_release": (ctypes.c_int, []),
    "fp_plan_count": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(PlanSizes)]),
    "fp_plan_fill": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.c_int, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "fp_plan_count_rule": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.POINTER(TileRule), ctypes.POINTER(PlanSizes)]),
    "fp_plan_fill_rule": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.POINTER(TileRule), c_vp, c_vp, c_vp, c_vp,
                                         c_vp]),
    "fp_plan_bbox": (ctypes.c_int, [c_vp, ctypes.POINTER(PlanSizes), ctypes.POINTER(PlanTables), c_vp]),
    "fp_plan_pack": (ctypes.c_int, [c_vp, ctypes.POINTER(PlanSizes), ctypes.POINTER(PlanTables), c_vp, c_vp]),
    "fp_tile_smem_bytes": (ctypes.c_int, [ctypes.c_int, c_i64, ctypes.POINTER(c_i64)]),
    "fp_evaluate_batch": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.POINTER(PlanSizes), ctypes.POINTER(PlanTables),
                                         c_vp, c_vp, c_vp, c_vp, c_sz, ctypes.POINTER(Launch), c_vp]),
    "fp_evaluate_batch_noalloc": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.POINTER(PlanSizes),
                                                 ctypes.POINTER(PlanTables), c_vp, c_vp, c_vp,
                                                 ctypes.POINTER(Launch), c_vp]),
    "fp_read_status": (ctypes.c_int, [c_vp, ctypes.POINTER(c_i32), c_vp]),
    "fp_read_status_noalloc": (ctypes.c_int, [ctypes.POINTER(c_i32), c_vp]),
    "fp_count_pairs": (ctypes.c_int, [c_vp, ctypes.POINTER(PlanSizes), ctypes.POINTER(PlanTables), c_vp, c_sz,
                                      c_vp, c_vp]),
    "fp_hmc_prepare": (ctypes.c_int, [c_vp, ctypes.c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "fp_hmc_lnprob": (ctypes.c_int, [c_vp, ctypes.c_int, c_vp, c_vp, c_vp, c_vp, ctypes.c_int, ctypes.c_int,
                                     c_vp, c_vp, c_vp]),
    "fp_hmc_leapfrog": (ctypes.c_int, [c_vp, ctypes.c_int, c_vp, ctypes.c_int, c_vp]),
    "fp_measure_peaks": (ctypes.c_int, [c_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                        c_vp]),
}


class NativeError(RuntimeError):
    pass


_lib = None


def lib_path():
    return _build.variant_lib() if _build.LIB == _build.DEFAULT_LIB else _build.LIB


def load(build_if_missing=True):
    """Load (building first if needed) the CUDA library and check its struct sizes."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if build_if_missing and path == _build.DEFAULT_LIB:
        _build.build()
    if not os.path.exists(path):
        raise NativeError("CUDA library %s is missing; run python -m forcepho_b200.build" % path)
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    sizes = np.zeros(4, dtype=np.int32)
    L.fp_struct_sizes(sizes.ctypes.data)
    want = [STRUCT_SIZES["patch"], STRUCT_SIZES["source"], STRUCT_SIZES["response"], STRUCT_SIZES["psf"]]
    if list(sizes) != want:
        raise NativeError("struct sizes of %s are %s, expected %s" % (path, list(sizes), want))
    _lib = L
    return L


def check(rc, what=""):
    """Raise NativeError with the library's message when rc != 0."""
    if rc != 0:
        msg = load().fp_error_string().decode(errors="replace")
        raise NativeError("%s failed (%d): %s" % (what, rc, msg))
    return rc


def patch_shape(patch, coordinates=True):
    """PatchShape of a PatchBase (with its pixel coordinates unless
    ``coordinates`` is False); keeps the arrays alive on the returned object."""
    keep = [np.ascontiguousarray(patch.exposure_start, dtype=np.int32),
            np.ascontiguousarray(patch.exposure_N, dtype=np.int32),
            np.ascontiguousarray(patch.band_start, dtype=np.int16),
            np.ascontiguousarray(patch.band_N, dtype=np.int16),
            np.ascontiguousarray(patch.n_psf_per_source, dtype=np.int32),
            np.ascontiguousarray(patch.xpix, dtype=np.float32),
            np.ascontiguousarray(patch.ypix, dtype=np.float32)]
    xp, yp = (keep[5].ctypes.data, keep[6].ctypes.data) if coordinates else (None, None)
    s = PatchShape(patch.n_bands, patch.n_exp, int(patch.n_sources), patch.npix,
                   keep[0].ctypes.data, keep[1].ctypes.data, keep[2].ctypes.data, keep[3].ctypes.data,
                   keep[4].ctypes.data, xp, yp)
    s._keep = keep
    return s
