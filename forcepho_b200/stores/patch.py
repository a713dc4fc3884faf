"""Patches packed from image stores: the input side of the batched kernel.

The reference builds every patch it samples from stored exposures
(forcepho/patches/pixel_patch.py:52-486, forcepho/patches/patch.py:222-500):
find the exposures that overlap a sky region, take the pixels of each inside
the region, pack them band by band into the 1-D pixel arrays (``pack_pix``),
and pack each scene's source metadata from the exposures' WCS and the PSF
store (``pack_meta``).  This module does the same, with the readers of this
package in place of astropy and h5py:

* ``FITSPatch``  -- exposures in FITS files (science extension, inverse
  uncertainty from the uncertainty extension), as the reference's FITSPatch;
* ``StorePatch`` -- exposures in a super-pixel HDF5 pixel store with a JSON
  header store (the reference's PixelStore / MetaStore layout,
  forcepho/patches/storage.py:43-430);
* ``PSFStore``   -- per-band PSF mixtures (forcepho/patches/storage.py:436-489).

Both patch classes carry the device mixin, so a packed patch goes straight
to ``send_to_device`` and into ``BatchedProposer`` or a ``PatchFarm`` work
list.  Source positions follow the reference's convention: ``set_scene``
takes absolute (ra, dec) degrees; ``pack_meta`` makes them offsets from the
patch reference coordinate (the scene's median position), as ``zerocoords``
does, and ``meta_for`` packs any scene given in those offsets.
"""

import json

import numpy as np

from ..device import B200PatchMixin
from ..patch import PatchBase
from ..sources import Galaxy, Scene
from ..splines import default_splines
from ..structs import psf_dtype
from . import fits as F
from .h5lite import H5File
from .wcs import TanWCS, scale_at_sky

__all__ = ["PSFStore", "MetaStore", "PixelStore", "StorePatchBase", "FITSPatch", "StorePatch", "JWST_BANDS"]

JWST_BANDS = ["F090W", "F115W", "F150W", "F200W", "F277W", "F335M", "F356W", "F410M", "F444W"]


class PSFStore:
    """Per-band PSF mixtures: ``band/parameters`` [n_loc, n_psf_per_source]
    records (amp, xcen, ycen, Cxx, Cyy, Cxy, sersic_bin) and the attribute
    ``n_psf_per_source`` of each band group; ``band/detector_locations``
    (optional) selects the record set nearest a source's pixel position."""

    def __init__(self, h5file):
        self.h5file = h5file
        self._f = H5File(h5file)
        self._cache = {}

    def n_psf_per_source(self, band):
        return int(self._f[band].attrs["n_psf_per_source"])

    def lookup(self, band, xy=None):
        if band not in self._cache:
            g = self._f[band]
            locs = g["detector_locations"].read() if "detector_locations" in g else None
            self._cache[band] = (g["parameters"].read(), locs)
        pars, locs = self._cache[band]
        choose = 0
        if xy is not None and locs is not None:
            xp, yp = locs
            choose = int(np.argmin(np.hypot(xy[0] - xp, xy[1] - yp)))
        return np.atleast_2d(pars)[choose]

    def get_local_psf(self, band, source=None, wcs=None):
        """The PSF records of one source in one band (n_psf_per_source rows)."""
        xy = None
        if wcs is not None and source is not None:
            xy = wcs.all_world2pix(source.ra, source.dec, 0)
        p = self.lookup(band, xy)
        out = np.zeros(len(p), dtype=psf_dtype)
        for c in ("amp", "xcen", "ycen", "Cxx", "Cyy", "Cxy"):
            out[c] = p[c]
        out["sersic_bin"] = p["sersic_bin"]
        return out


def _header_from_string(s):
    """A FITS header serialised as 80-character cards (the MetaStore's JSON values)."""
    h = {}
    for j in range(0, len(s), F.CARD):
        card = s[j:j + F.CARD]
        key = card[:8].strip()
        if key == "END":
            break
        if card[8:10] == "= " and key:
            h[key] = F._value(card[10:])
    return h


class MetaStore:
    """Exposure headers by band and exposure id (JSON of serialised FITS
    headers, as forcepho/patches/storage.py:285-366 writes it), with a WCS per
    exposure."""

    def __init__(self, metastorefile=None):
        self.headers, self.wcs = {}, {}
        if metastorefile:
            with open(metastorefile) as f:
                raw = json.load(f)
            for band, exps in raw.items():
                self.headers[band] = {e: _header_from_string(h) for e, h in exps.items()}
            for band, exps in self.headers.items():
                self.wcs[band] = {e: TanWCS(h) for e, h in exps.items()}


class PixelStore:
    """Super-pixel store: ``band/expID/data`` arrays of shape
    (nsuper, nsuper, 2 s^2) holding each super-pixel's s x s fluxes then
    inverse errors; root attributes ``nside_full`` and ``super_pixel_size``."""

    def __init__(self, h5file):
        self.h5file = h5file
        self._f = H5File(h5file)
        a = self._f.attrs
        self.nside_full = np.zeros(2, dtype=np.int64) + np.asarray(a["nside_full"])
        self.super_pixel_size = int(a["super_pixel_size"])
        self.xpix, self.ypix = self.pixel_coordinates()

    def superpixelize(self, a, b):
        s = self.super_pixel_size
        nx, ny = (np.array(a.shape) // s).astype(int)
        ta = a[:nx * s, :ny * s].reshape(nx, s, ny, s).transpose(0, 2, 1, 3).reshape(nx, ny, s * s)
        tb = b[:nx * s, :ny * s].reshape(nx, s, ny, s).transpose(0, 2, 1, 3).reshape(nx, ny, s * s)
        return np.concatenate([ta, tb], axis=-1)

    def pixel_coordinates(self):
        yy, xx = np.meshgrid(np.arange(self.nside_full[1]), np.arange(self.nside_full[0]))
        packed = self.superpixelize(xx, yy)
        s2 = self.super_pixel_size ** 2
        return packed[:, :, :s2].astype(np.int16), packed[:, :, s2:].astype(np.int16)

    def superpixel_corners(self):
        lower_left = np.array([self.xpix[:, :, 0], self.ypix[:, :, 0]])
        offsets = np.array([(0, 0), (1, 0), (1, 1), (0, 1)]) * (self.super_pixel_size - 1)
        corners = offsets[:, :, None, None] + lower_left[None, :, :, :]
        return corners.transpose(2, 3, 0, 1)

    def data(self, epath):
        return self._f[epath + "/data"].read()


class StorePatchBase(B200PatchMixin, PatchBase):
    """Pixel packing and metadata packing shared by the store-backed patches
    (forcepho/patches/pixel_patch.py:52-209, forcepho/patches/patch.py:222-470).
    Subclasses give ``find_exposures`` and ``find_pixels``."""

    def __init__(self, psfstore="", splinedata=None, return_residual=False, meta_dtype=np.float32,
                 pix_dtype=np.float32, debug=0):
        super().__init__(return_residual=return_residual, pix_dtype=pix_dtype, meta_dtype=meta_dtype)
        self.psfstore = PSFStore(psfstore) if psfstore else None
        self.splines = splinedata if splinedata is not None else default_splines()
        self.debug = debug
        self.patch_reference_coordinates = np.zeros(2)
        self.wcs_origin = 0
        self.background_offsets = None
        self.max_snr = None
        self.scene = None

    # --- pixels ---
    def build_patch(self, region=None, sourcecat=None, allbands=JWST_BANDS, tweak_background=False):
        """Find the exposures overlapping ``region`` and pack their pixels
        inside it (band by band); with ``sourcecat`` also set and pack its
        scene (pixel_patch.py:52-123)."""
        self.hdrs, self.wcses, self.epaths, self.bands = self.find_exposures(region, allbands)
        if len(self.epaths) == 0:
            raise ValueError("No exposures in the specified bands overlap the region")
        self.background_offsets = ([h.get(tweak_background, 0.0) for h in self.hdrs]
                                   if tweak_background else None)
        allbands = list(allbands)
        band_ids = [allbands.index(b) for b in self.bands]
        if np.any(np.diff(band_ids) < 0):
            raise ValueError("exposures must be sorted by band")
        u, n = np.unique(band_ids, return_counts=True)
        self.uniq_bands, self.n_exp_per_band = u, n
        self.bandlist = [allbands[i] for i in self.uniq_bands]
        self.pack_pix(region)
        if sourcecat is not None:
            self.pack_meta(self.set_scene(sourcecat))
        self._dirty_data = False

    def pack_pix(self, region):
        """Concatenate the exposures' pixels into the 1-D arrays and fill the
        band / exposure index arrays (pixel_patch.py:125-196)."""
        nb, ne = len(self.bandlist), len(self.hdrs)
        self.band_start = np.empty(nb, dtype=np.int16)
        self.band_N = np.zeros(nb, dtype=np.int16)
        self.exposure_start = np.empty(ne, dtype=np.int32)
        self.exposure_N = np.empty(ne, dtype=np.int32)
        data, ierr, xpix, ypix = [], [], [], []
        b, i = 0, 0
        for e, wcs in enumerate(self.wcses):
            d, ie, xp, yp = self.find_pixels(self.epaths[e], wcs, region)
            n_pix = d.size
            if n_pix == 0:
                raise ValueError("There were no valid pixels in exposure %s" % self.epaths[e])
            if self.background_offsets is not None:
                d = d - self.background_offsets[e]
            if e > 0 and self.bands[e] != self.bands[e - 1]:
                b += 1
            self.band_N[b] += 1
            self.exposure_start[e] = i
            self.exposure_N[e] = n_pix
            data.append(np.ravel(d))
            ierr.append(np.ravel(ie))
            xpix.append(np.ravel(xp))
            ypix.append(np.ravel(yp))
            i += n_pix
        dt = self.pix_dtype
        self.data = np.concatenate(data).astype(dt)
        self.ierr = np.concatenate(ierr).astype(dt)
        self.xpix = np.concatenate(xpix).astype(dt)
        self.ypix = np.concatenate(ypix).astype(dt)
        self.band_start[0] = 0
        self.band_start[1:] = np.cumsum(self.band_N)[:-1]
        if self.max_snr:
            cap = (self.ierr > 0) & (self.data * self.ierr > self.max_snr)
            self.ierr[cap] = self.max_snr / self.data[cap]

    # --- scenes and metadata ---
    def set_scene(self, sourcecat, splinedata=None):
        """A Scene of Galaxy sources from a catalog with ra, dec (absolute
        degrees), q, pa, sersic, rhalf and one flux column per band of
        ``bandlist`` (patch.py:400-425)."""
        splines = splinedata if splinedata is not None else self.splines
        scene = Scene()
        for row in np.atleast_1d(sourcecat):
            g = Galaxy(filternames=self.bandlist, splines=splines)
            g.flux[:] = [float(row[b]) for b in self.bandlist]
            g.ra, g.dec = float(row["ra"]), float(row["dec"])
            g.q, g.pa = float(row["q"]), float(row["pa"])
            g.sersic, g.rhalf = float(row["sersic"]), float(row["rhalf"])
            scene.sources.append(g)
        return scene

    def zerocoords(self, scene, sky_zero=None):
        """Make the scene's positions offsets from a reference coordinate (the
        median source position unless given), in place, so that FP32
        proposals keep their precision (patch.py:427-461)."""
        if sky_zero is None:
            if len(scene.sources) == 0:
                sky_zero = self.patch_reference_coordinates
            else:
                sky_zero = np.array([np.median([s.ra for s in scene.sources]),
                                     np.median([s.dec for s in scene.sources])])
        zero = np.array(sky_zero, dtype=np.float64)
        self.patch_reference_coordinates = zero
        for s in scene.sources:
            s.ra -= zero[0]
            s.dec -= zero[1]
        return zero

    def meta_for(self, scene):
        """Source metadata of a scene whose positions are offsets from the
        patch reference coordinate (patch.py:274-398): D, CW, crpix, crval
        per exposure and source, the PSF records of every (exposure, source),
        without changing the patch."""
        srcs = list(scene.sources)
        ns, ne = len(srcs), len(self.wcses)
        dt = self.meta_dtype
        ra0, dec0 = self.patch_reference_coordinates
        D = np.empty((ne, ns, 2, 2), dtype=dt)
        CW = np.empty((ne, ns, 2, 2), dtype=dt)
        crpix = np.empty((ne, ns, 2), dtype=dt)
        crval = np.empty((ne, ns, 2), dtype=dt)
        for j, wcs in enumerate(self.wcses):
            for i, s in enumerate(srcs):
                ssky = np.array([s.ra + ra0, s.dec + dec0])
                CW_mat, D_mat = scale_at_sky(ssky, wcs)
                D[j, i], CW[j, i] = D_mat, CW_mat
                crval[j, i] = ssky - self.patch_reference_coordinates
                crpix[j, i] = wcs.all_world2pix(ssky[0], ssky[1], self.wcs_origin)
        npsf = np.array([self.psfstore.n_psf_per_source(b) for b in self.bandlist], dtype=np.int32)
        pstart = np.zeros(ne, dtype=np.int32)
        blocks, k = [], 0
        for e in range(ne):
            pstart[e] = k
            for s in srcs:
                p = self.psfstore.get_local_psf(band=self.bands[e], source=s)
                blocks.append(p)
                k += len(p)
        psfgauss = np.concatenate(blocks) if blocks else np.zeros(0, psf_dtype)
        rad2 = (np.asarray(srcs[0].radii, np.float64) ** 2).astype(dt) if srcs else \
            (np.asarray(self.splines.radii, np.float64) ** 2).astype(dt)
        return dict(n_sources=ns, n_radii=len(rad2), rad2=rad2, D=D, CW=CW, crpix=crpix, crval=crval,
                    G=np.ones(ne, dtype=dt), n_psf_per_source=npsf, psfgauss=psfgauss, psfgauss_start=pstart)

    def pack_meta(self, scene):
        """Make ``scene`` the patch's scene: zero its coordinates and pack its
        metadata (patch.py:244-272); the pixels are untouched."""
        self.zerocoords(scene)
        for k, v in self.meta_for(scene).items():
            setattr(self, k, v)
        self.scene = scene

    def catalog(self, scene=None):
        """The structured catalog of a scene in absolute coordinates (the
        inverse of ``set_scene``)."""
        scene = scene if scene is not None else self.scene
        dt = np.dtype([(c, np.float64) for c in ("ra", "dec", "q", "pa", "sersic", "rhalf")] +
                      [(b, np.float64) for b in self.bandlist])
        cat = np.zeros(len(scene.sources), dtype=dt)
        ra0, dec0 = self.patch_reference_coordinates
        for i, g in enumerate(scene.sources):
            cat[i]["ra"], cat[i]["dec"] = g.ra + ra0, g.dec + dec0
            cat[i]["q"], cat[i]["pa"], cat[i]["sersic"], cat[i]["rhalf"] = g.q, g.pa, g.sersic, g.rhalf
            for j, b in enumerate(self.bandlist):
                cat[i][b] = g.flux[j]
        return cat


class FITSPatch(StorePatchBase):
    """Exposures in FITS files: the science image in extension ``sci_ext``
    and its uncertainty in ``unc_ext`` (pixel_patch.py:356-486); pixels
    outside the region are dropped, non-finite or negative inverse errors
    masked, and each exposure padded to ``warp_size`` pixels with ierr = 0
    and x = y = -1."""

    warp_size = 64

    def __init__(self, fitsfiles=(), psfstore="", splinedata=None, return_residual=False, sci_ext=0, unc_ext=1,
                 meta_dtype=np.float32, pix_dtype=np.float32, debug=0):
        super().__init__(psfstore=psfstore, splinedata=splinedata, return_residual=return_residual,
                         meta_dtype=meta_dtype, pix_dtype=pix_dtype, debug=debug)
        self.fitsfiles = list(fitsfiles) if not isinstance(fitsfiles, str) else [fitsfiles]
        self.sci_ext, self.unc_ext = sci_ext, unc_ext
        self.snr = None
        self.unc = None
        self._hdus = {}

    def _read(self, path):
        if path not in self._hdus:
            self._hdus[path] = F.read_fits(path)
        return self._hdus[path]

    def find_exposures(self, region, bandlist, do_check=True):
        imbands = [str(self._read(f)[self.sci_ext].header.get("FILTER", "")).strip() for f in self.fitsfiles]
        epaths, bands, hdrs, wcses = [], [], [], []
        for band in bandlist:
            for path, b in zip(self.fitsfiles, imbands):
                if b != band:
                    continue
                hdr = self._read(path)[self.sci_ext].header
                wcs = TanWCS(hdr)
                if region is not None and do_check:
                    bra, bdec = region.bounding_box
                    nx, ny = hdr["NAXIS1"], hdr["NAXIS2"]
                    bx, by = wcs.all_world2pix(bra, bdec, self.wcs_origin)
                    inim = np.any((bx > 0) & (bx < nx) & (by > 0) & (by < ny))
                    around = (nx < bx.max()) & (bx.min() < 0) & (ny < by.max()) & (by.min() < 0)
                    if not (inim or around):
                        continue
                epaths.append(path)
                wcses.append(wcs)
                bands.append(b)
                hdrs.append(hdr)
        return hdrs, wcses, epaths, bands

    def find_pixels(self, epath, wcs, region):
        hdus = self._read(epath)
        flux = np.array(hdus[self.sci_ext].data, dtype=np.float64).T        # (x, y) order
        if self.snr is not None:
            ie = self.snr / flux
        elif self.unc is not None:
            ie = np.zeros_like(flux) + 1.0 / self.unc
        else:
            with np.errstate(divide="ignore"):
                ie = 1.0 / np.array(hdus[self.unc_ext].data, dtype=np.float64).T
        bad = ~np.isfinite(flux) | ~np.isfinite(ie) | (ie < 0)
        ie[bad] = 0
        flux[bad] = 0
        nx, ny = flux.shape
        yp, xp = np.meshgrid(np.arange(ny), np.arange(nx))
        if region is None:
            sx, sy = slice(None), slice(None)
        else:
            offsets = np.array([(0, 0), (1, 0), (1, 1), (0, 1)])
            lower_left = np.array([xp, yp])
            corners = (offsets[:, :, None, None] + lower_left[None, :, :, :]).transpose(2, 3, 0, 1)
            sx, sy = region.contains(corners[..., 0], corners[..., 1], wcs, origin=self.wcs_origin)
        flux, ie = flux[sx, sy].reshape(-1), ie[sx, sy].reshape(-1)
        xp, yp = xp[sx, sy].reshape(-1), yp[sx, sy].reshape(-1)
        pad = (-len(flux)) % self.warp_size
        if pad:
            flux = np.append(flux, np.zeros(pad))
            ie = np.append(ie, np.zeros(pad))
            xp = np.append(xp, np.zeros(pad) - 1)
            yp = np.append(yp, np.zeros(pad) - 1)
        return flux, ie, xp, yp


class StorePatch(StorePatchBase):
    """Exposures in a super-pixel HDF5 pixel store with a JSON header store
    (pixel_patch.py:212-353): super-pixels with a corner inside the region."""

    def __init__(self, pixelstore="", metastore="", psfstore="", splinedata=None, return_residual=False,
                 meta_dtype=np.float32, pix_dtype=np.float32, debug=0):
        super().__init__(psfstore=psfstore, splinedata=splinedata, return_residual=return_residual,
                         meta_dtype=meta_dtype, pix_dtype=pix_dtype, debug=debug)
        self.metastore = MetaStore(metastore)
        self.pixelstore = PixelStore(pixelstore)

    def find_exposures(self, region, bandlist):
        imsize = np.zeros(2) + self.pixelstore.nside_full
        corners = self.pixelstore.superpixel_corners()
        bra, bdec = region.bounding_box
        epaths, bands, hdrs, wcses = [], [], [], []
        for band in bandlist:
            if band not in self.metastore.wcs:
                continue
            for expID, wcs in self.metastore.wcs[band].items():
                bx, by = wcs.all_world2pix(bra, bdec, self.wcs_origin)
                if not np.any((bx > 0) & (bx < imsize[0]) & (by > 0) & (by < imsize[1])):
                    continue
                sx, _ = region.contains(corners[..., 0], corners[..., 1], wcs, origin=self.wcs_origin)
                if len(sx) == 0:
                    continue
                wcses.append(wcs)
                epaths.append("%s/%s" % (band, expID))
                bands.append(band)
                hdrs.append(self.metastore.headers[band][expID])
        return hdrs, wcses, epaths, bands

    def find_pixels(self, epath, wcs, region):
        s2 = self.pixelstore.super_pixel_size ** 2
        corners = self.pixelstore.superpixel_corners()
        sx, sy = region.contains(corners[..., 0], corners[..., 1], wcs, origin=self.wcs_origin)
        data = self.pixelstore.data(epath)
        return (data[sx, sy, :s2], data[sx, sy, s2:], self.pixelstore.xpix[sx, sy, :],
                self.pixelstore.ypix[sx, sy, :])
