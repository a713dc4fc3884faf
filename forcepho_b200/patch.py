"""Patch data model: pixel and metadata arrays of one sky patch.

``PatchBase`` holds the same arrays, with the same shapes, dtypes and packing
conventions, as the reference's ``PatchBase.build_patch`` documents
(forcepho/patches/patch.py:122-198):

* pixels of all exposures concatenated in band order, each exposure padded to
  a multiple of 32 pixels (pad pixels carry ierr = 0):
  ``xpix, ypix, data, ierr`` f32[npix];
* ``exposure_start, exposure_N`` i32[n_exp]; ``band_start, band_N`` i16[n_bands];
* ``n_sources``, ``n_radii``, ``rad2`` f32[n_radii];
* ``D, CW`` f32[n_exp, n_sources, 2, 2]; ``crpix, crval`` f32[n_exp, n_sources, 2];
  ``G`` f32[n_exp];
* ``n_psf_per_source`` i32[n_bands]; ``psfgauss`` psf_dtype[sum_e n_sources *
  n_psf_per_source[band(e)]]; ``psfgauss_start`` i32[n_exp].

The device side (``forcepho_b200.device.B200PatchMixin``) mirrors the
reference's ``GPUPatchMixin`` on top of these arrays.
"""

import numpy as np

from .structs import patch_struct_dtype, psf_dtype, meta_names

__all__ = ["PatchBase"]

PIXEL_NAMES = ["data", "ierr", "xpix", "ypix"]
INDEX_NAMES = ["exposure_start", "exposure_N", "band_start", "band_N"]


class PatchBase:
    """Host-side container of one patch's arrays (see module docstring)."""

    patch_struct_dtype = patch_struct_dtype
    meta_names = meta_names

    def __init__(self, return_residual=False, pix_dtype=np.float32, meta_dtype=np.float32):
        self.pix_dtype = pix_dtype
        self.meta_dtype = meta_dtype
        self.return_residual = return_residual
        self._dirty_data = True

    # --- shapes ---
    @property
    def npix(self):
        x = getattr(self, "xpix", None)
        return 0 if x is None else int(x.shape[0])

    @property
    def n_bands(self):
        return int(len(self.band_N))

    @property
    def n_exp(self):
        return int(len(self.exposure_N))

    @property
    def band_N_pix(self):
        """Pixels (with padding) in each band."""
        out = np.zeros(self.n_bands, dtype=np.int64)
        for b in range(self.n_bands):
            e0, ne = int(self.band_start[b]), int(self.band_N[b])
            out[b] = int(np.sum(self.exposure_N[e0:e0 + ne]))
        return out

    def exposure_band(self):
        """Sequential band index of every exposure."""
        eb = np.empty(self.n_exp, dtype=np.int32)
        for b in range(self.n_bands):
            e0, ne = int(self.band_start[b]), int(self.band_N[b])
            eb[e0:e0 + ne] = b
        return eb

    def n_gauss_per_exposure(self):
        return int(self.n_sources) * self.n_psf_per_source[self.exposure_band()].astype(np.int64)

    def max_gauss_per_exposure(self):
        return int(int(self.n_sources) * int(np.max(self.n_psf_per_source)))

    def n_pairs(self):
        """(pixel, image Gaussian) pairs per likelihood evaluation."""
        return int(np.sum(self.exposure_N.astype(np.int64) * self.n_gauss_per_exposure()))

    def build_patch(self, npix=1, n_sources=1, n_radii=1, n_bands=1, n_exp=1):
        """Allocate empty arrays of the documented shapes (forcepho/patches/patch.py:122-198)."""
        self.xpix = np.zeros(npix, dtype=self.pix_dtype)
        self.ypix = np.zeros(npix, dtype=self.pix_dtype)
        self.data = np.zeros(npix, dtype=self.pix_dtype)
        self.ierr = np.zeros(npix, dtype=self.pix_dtype)
        self.band_start = np.zeros(n_bands, dtype=np.int16)
        self.band_N = np.zeros(n_bands, dtype=np.int16)
        self.exposure_start = np.zeros(n_exp, dtype=np.int32)
        self.exposure_N = np.zeros(n_exp, dtype=np.int32)
        self.n_sources = n_sources
        self.n_radii = n_radii
        self.rad2 = np.zeros(n_radii, dtype=self.meta_dtype)
        self.D = np.zeros((n_exp, n_sources, 2, 2), dtype=self.meta_dtype)
        self.CW = np.zeros((n_exp, n_sources, 2, 2), dtype=self.meta_dtype)
        self.crpix = np.zeros((n_exp, n_sources, 2), dtype=self.meta_dtype)
        self.crval = np.zeros((n_exp, n_sources, 2), dtype=self.meta_dtype)
        self.G = np.ones(n_exp, dtype=self.meta_dtype)
        self.n_psf_per_source = np.zeros(n_bands, dtype=np.int32)
        self.psfgauss = np.zeros(0, dtype=psf_dtype)
        self.psfgauss_start = np.zeros(n_exp, dtype=np.int32)

    def validate(self):
        """Host-side checks of the index arrays before anything is sent to a device.

        Raises ValueError on the first inconsistency (the reference kernel has
        no such checks and would read out of bounds instead)."""
        from .kernel_limits import MAXBANDS, MAXSOURCES, MAXRADII
        n_b, n_e, n_s = self.n_bands, self.n_exp, int(self.n_sources)
        if not (1 <= n_b <= MAXBANDS):
            raise ValueError(f"n_bands={n_b} outside [1, {MAXBANDS}]")
        if not (0 <= n_s <= MAXSOURCES):
            raise ValueError(f"n_sources={n_s} outside [0, {MAXSOURCES}]")
        if not (1 <= int(self.n_radii) <= MAXRADII) or len(self.rad2) != int(self.n_radii):
            raise ValueError("rad2 / n_radii inconsistent or above MAXRADII")
        bs, bn = self.band_start.astype(np.int64), self.band_N.astype(np.int64)
        if np.any(bn < 0) or bs[0] != 0 or np.any(bs[1:] != np.cumsum(bn)[:-1]) or bn.sum() != n_e:
            raise ValueError("band_start/band_N do not tile the exposures in order")
        es, en = self.exposure_start.astype(np.int64), self.exposure_N.astype(np.int64)
        if np.any(en < 0) or np.any(es < 0) or np.any(es + en > self.npix):
            raise ValueError("exposure_start/exposure_N exceed the pixel arrays")
        for name in ["ypix", "data", "ierr"]:
            if getattr(self, name).shape != self.xpix.shape:
                raise ValueError(f"{name} shape differs from xpix")
        for name, shp in [("D", (n_e, n_s, 2, 2)), ("CW", (n_e, n_s, 2, 2)),
                          ("crpix", (n_e, n_s, 2)), ("crval", (n_e, n_s, 2))]:
            if getattr(self, name).shape != shp:
                raise ValueError(f"{name} has shape {getattr(self, name).shape}, expected {shp}")
        if len(self.G) != n_e or len(self.psfgauss_start) != n_e or len(self.n_psf_per_source) != n_b:
            raise ValueError("G / psfgauss_start / n_psf_per_source lengths inconsistent")
        eb = self.exposure_band()
        npsf = self.n_psf_per_source[eb].astype(np.int64)
        if np.any(npsf <= 0):
            raise ValueError("n_psf_per_source must be positive")
        # with no sources the PSF blocks are never read (and are empty)
        if n_s > 0 and np.any(self.psfgauss_start.astype(np.int64) + npsf > len(self.psfgauss)):
            raise ValueError("psfgauss_start + n_psf_per_source exceeds psfgauss")
        bins = self.psfgauss["sersic_bin"]
        if len(bins) and (bins.min() < 0 or bins.max() >= int(self.n_radii)):
            raise ValueError("psfgauss sersic_bin outside [0, n_radii)")
        return True

    def split_pix(self, attr):
        arr = getattr(self, attr)
        return np.split(arr, np.cumsum(self.exposure_N[:-1]))

    def split_band(self, attr):
        """A pixel array split by band (forcepho/patches/patch.py:610-620)."""
        arr = getattr(self, attr)
        return np.split(arr, np.cumsum(self.band_N_pix[:-1]))
