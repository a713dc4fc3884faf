"""numpy dtypes of the records that cross the host/device boundary.

Each dtype is byte-identical to the reference's so that arrays packed by the
reference's Python code can be handed to this library unchanged:

* ``source_struct_dtype``   -- forcepho/proposal.py:229-240 (264 bytes)
* ``response_struct_dtype`` -- forcepho/proposal.py:242-244 (840 bytes)
* ``patch_struct_dtype``    -- forcepho/patches/patch.py:44-73 (152 bytes)
* ``psf_dtype``             -- forcepho/patches/storage.py:26-28 (28 bytes)

and to the C structs of ``include/forcepho_b200.h`` (checked against
``fp_struct_sizes`` when the library loads).
"""

import numpy as np

from .kernel_limits import MAXBANDS, MAXRADII, MAXSOURCES, NPARAMS

source_float_dt = np.float32

source_struct_dtype = np.dtype([("ra", source_float_dt),
                                ("dec", source_float_dt),
                                ("q", source_float_dt),
                                ("pa", source_float_dt),
                                ("nsersic", source_float_dt),
                                ("rh", source_float_dt),
                                ("fluxes", source_float_dt, MAXBANDS),
                                ("mixture_amplitudes", source_float_dt, MAXRADII),
                                ("damplitude_drh", source_float_dt, MAXRADII),
                                ("damplitude_dnsersic", source_float_dt, MAXRADII)],
                               align=True)

response_float_dt = source_float_dt
response_struct_dtype = np.dtype([("dchi2_dparam", response_float_dt,
                                   NPARAMS * MAXSOURCES)], align=True)

ptr_dtype = np.uintp
patch_struct_dtype = np.dtype([("data", ptr_dtype),
                               ("ierr", ptr_dtype),
                               ("xpix", ptr_dtype),
                               ("ypix", ptr_dtype),
                               ("residual", ptr_dtype),
                               ("exposure_start", ptr_dtype),
                               ("exposure_N", ptr_dtype),
                               ("band_start", ptr_dtype),
                               ("band_N", ptr_dtype),
                               ("n_sources", np.int32),
                               ("n_radii", np.int32),
                               ("rad2", ptr_dtype),
                               ("D", ptr_dtype),
                               ("crpix", ptr_dtype),
                               ("crval", ptr_dtype),
                               ("CW", ptr_dtype),
                               ("G", ptr_dtype),
                               ("n_psf_per_source", ptr_dtype),
                               ("psfgauss", ptr_dtype),
                               ("psfgauss_start", ptr_dtype)],
                              align=True)

PSF_COLS = ["amp", "xcen", "ycen", "Cxx", "Cyy", "Cxy"]
psf_dtype = np.dtype([(c, np.float32) for c in PSF_COLS] + [("sersic_bin", np.int32)])

# Names of the patch-struct fields that are pointers to metadata arrays
# (the ones re-sent when the scene changes), forcepho/patches/patch.py:76-78.
meta_names = ["n_sources", "n_radii", "rad2", "D", "crpix", "crval", "CW", "G",
              "n_psf_per_source", "psfgauss", "psfgauss_start"]

# (dtype, itemsize the C side reports) for the load-time check.
STRUCT_SIZES = {"patch": 152, "source": 264, "response": 840, "psf": 28}

assert patch_struct_dtype.itemsize == STRUCT_SIZES["patch"]
assert source_struct_dtype.itemsize == STRUCT_SIZES["source"]
assert response_struct_dtype.itemsize == STRUCT_SIZES["response"]
assert psf_dtype.itemsize == STRUCT_SIZES["psf"]

__all__ = ["source_struct_dtype", "response_struct_dtype", "patch_struct_dtype",
           "psf_dtype", "PSF_COLS", "meta_names", "ptr_dtype", "STRUCT_SIZES"]
