"""Seeded synthetic patches for the five workloads of this hot path.

No survey data is available offline, so every workload is a synthetic patch
with the layout a real forcepho patch has (``PatchBase``): pixel scale 0.03"
per pixel, linear per-exposure astrometry expressed as the reference's ``D``
(pix/arcsec) and ``CW`` (pix/deg) matrices (forcepho/patches/patch.py:504-560),
source positions stored as degree offsets from a patch reference coordinate
(patch.py:427-461), ``G = 1``, the 9 Sersic radii of the reference's spline
table, PSF mixtures replicated across the radius bins with ``sersic_bin = r``
(demo/demo_utils.py:212-230), raster pixel order, exposures padded to a
multiple of 32 pixels with ierr = 0 in the pad (xpix = ypix = -1 there, as
FITSPatch.find_pixels does, forcepho/patches/pixel_patch.py:473-484).

The workloads (``configs``):

* ``small``  -- 1 band x 1 exposure, 64x64 px, 1 source at the centre +- U(-2,2) px,
  flux 10, q 0.7, pa 0.4, sersic 2, rhalf 0.15"; PSF 3 isotropic Gaussians,
  Dirichlet(1) amplitudes, sigma U[0.8,3] px; noise sigma 1.
* ``multiband`` -- 5 bands x 2 exposures, 150x150 px, 16 sources uniform in the
  region; flux log-U(1,100) per band, q U(.3,.95), pa U(-pi/2,pi/2),
  sersic U(1,5), rhalf U(.05,.5)"; PSF 4 anisotropic Gaussians per band;
  small random rotation/shear per exposure; noise sigma U(.5,2) per exposure.
* ``limits`` -- 30 sources, 8 bands x 4 exposures, 256x256 px, 6-Gaussian PSFs,
  distributions as ``multiband``.
* ``batched`` -- 512 patches: sources U{1..30}, bands U{1..8}, exposures per band
  U{1..4}, pixels per exposure U{32^2..256^2} (the first n pixels of a 256-wide
  raster), PSFs as ``multiband``.
* ``hmc`` -- patches drawn like ``limits``.

Data pixels are the model rendered by a caller-supplied ``render(patch,
proposal) -> model`` (the GPU kernel in benchmarks, the oracle in tests) plus
Gaussian noise; with no renderer they are noise only.
"""

import numpy as np

from .device import B200PatchMixin
from .patch import PatchBase
from .sources import Galaxy, Scene
from .splines import default_splines
from .structs import psf_dtype

PIXSCALE = 0.03                      # arcsec per pixel
REF_COORD = np.array([53.1, -27.8])  # patch reference (ra, dec), degrees
PAD = 32

__all__ = ["make_patch", "config_small", "config_multiband", "config_limits",
           "config_batched", "config_hmc", "add_noise", "SyntheticPatch", "CONFIGS"]


class SyntheticPatch(B200PatchMixin, PatchBase):
    """A PatchBase (with the device mixin) carrying the scene it was drawn from.

    Like the reference's store-backed patches (forcepho/patches/patch.py:244-425)
    it keeps what is needed to pack the source metadata of any scene over the
    same pixels: each exposure's linear astrometry (``astrometry``: pixel =
    cen_e + A_e arcsec-offset) and PSF block (``psf_blocks``), with
    ``meta_for`` / ``pack_meta`` / ``set_scene``."""

    def __init__(self, **kw):
        super().__init__(**kw)
        self.scene = None
        self.sigma = None
        self.bandlist = None
        self.astrometry = None
        self.psf_blocks = None
        self.splines = None

    def meta_for(self, scene):
        """The source-dependent metadata arrays of ``scene`` (its sources in
        order) over this patch's exposures, without changing the patch:
        ``n_sources, D, CW, crpix, crval, psfgauss, psfgauss_start``."""
        A, cen = self.astrometry
        srcs = list(scene.sources)
        ns, ne = len(srcs), self.n_exp
        dt = self.meta_dtype
        D = np.zeros((ne, ns, 2, 2), dtype=dt)
        CW = np.zeros((ne, ns, 2, 2), dtype=dt)
        crpix = np.zeros((ne, ns, 2), dtype=dt)
        crval = np.zeros((ne, ns, 2), dtype=dt)
        for e in range(ne):
            for s, g in enumerate(srcs):
                cosd = np.cos(np.deg2rad(REF_COORD[1] + g.dec))
                W = np.diag([cosd, 1.0])
                D[e, s] = A[e]
                CW[e, s] = 3600.0 * A[e] @ W
                crval[e, s] = [g.ra, g.dec]
                crpix[e, s] = cen[e] + A[e] @ (3600.0 * W @ np.array([g.ra, g.dec]))
        # every source of an exposure gets a copy of the exposure's PSF block
        blocks, pstart, k = [], [], 0
        for e in range(ne):
            one = self.psf_blocks[e]
            pstart.append(k)
            for _ in range(ns):
                blocks.append(one)
                k += len(one)
        psfgauss = np.concatenate(blocks) if blocks else np.zeros(0, psf_dtype)
        return dict(n_sources=ns, D=D, CW=CW, crpix=crpix, crval=crval, psfgauss=psfgauss,
                    psfgauss_start=np.asarray(pstart, dtype=np.int32))

    def pack_meta(self, scene):
        """Make ``scene`` the patch's scene: repack its source metadata
        (forcepho/patches/patch.py:244-272); pixels are untouched."""
        for k, v in self.meta_for(scene).items():
            setattr(self, k, v)
        self.scene = scene

    def set_scene(self, sourcecat, splinedata=None):
        """A Scene of Galaxy sources from a structured catalog with fields
        ``ra, dec, q, pa, sersic, rhalf`` (ra/dec as degree offsets from the
        patch reference coordinate) and one flux field per name in
        ``bandlist`` (forcepho/patches/patch.py:400-425)."""
        splines = splinedata if splinedata is not None else self.splines
        scene = Scene()
        for row in np.atleast_1d(sourcecat):
            g = Galaxy(filternames=self.bandlist, splines=splines)
            g.flux[:] = [float(row[b]) for b in self.bandlist]
            g.ra, g.dec = float(row["ra"]), float(row["dec"])
            g.q, g.pa, g.sersic, g.rhalf = (float(row["q"]), float(row["pa"]), float(row["sersic"]),
                                            float(row["rhalf"]))
            scene.sources.append(g)
        return scene

    def catalog(self, scene=None):
        """The structured catalog of a scene (default: the patch's), the inverse of ``set_scene``."""
        scene = scene if scene is not None else self.scene
        dt = np.dtype([(c, np.float64) for c in ("ra", "dec", "q", "pa", "sersic", "rhalf")] +
                      [(b, np.float64) for b in self.bandlist])
        cat = np.zeros(len(scene.sources), dtype=dt)
        for i, g in enumerate(scene.sources):
            cat[i]["ra"], cat[i]["dec"] = g.ra, g.dec
            cat[i]["q"], cat[i]["pa"], cat[i]["sersic"], cat[i]["rhalf"] = g.q, g.pa, g.sersic, g.rhalf
            for j, b in enumerate(self.bandlist):
                cat[i][b] = g.flux[j]
        return cat


def _rot(t):
    c, s = np.cos(t), np.sin(t)
    return np.array([[c, -s], [s, c]])


def _psf_mixture(rng, n_p, anisotropic, offsets):
    """Amplitudes, centres and covariances (pixels) of one PSF mixture."""
    amps = rng.dirichlet(np.ones(n_p))
    cen = rng.uniform(-0.2, 0.2, (n_p, 2)) if offsets else np.zeros((n_p, 2))
    cov = np.empty((n_p, 2, 2))
    for i in range(n_p):
        sig = rng.uniform(0.8, 3.0)
        if anisotropic:
            ratio = rng.uniform(0.6, 1.0)
            R = _rot(rng.uniform(0, np.pi))
            cov[i] = R @ np.diag([sig ** 2, (sig * ratio) ** 2]) @ R.T
        else:
            cov[i] = np.eye(2) * sig ** 2
    return amps, cen, cov


def make_patch(rng, *, n_sources, exp_per_band, exp_pix, n_psf, psf_anisotropic=True,
               psf_offsets=True, perturb_wcs=True, source_params=None, splines=None,
               raster_width=None):
    """Draw one synthetic patch.

    Parameters
    ----------
    exp_per_band : list of int
        Exposures in each band.
    exp_pix : list of (width, height) or int
        Per exposure either a full ``width x height`` raster or, with
        ``raster_width`` set, an int: the first n pixels of a raster that wide.
    source_params : callable(rng, n_bands) -> dict or None
        Draws one source's ``flux`` array and ``q, pa, sersic, rhalf``;
        positions are drawn here, uniform in the first exposure's area.
    """
    splines = splines or default_splines()
    n_bands = len(exp_per_band)
    n_exp = int(sum(exp_per_band))
    radii = splines.radii
    n_radii = len(radii)
    band_of_exp = np.repeat(np.arange(n_bands), exp_per_band)

    # --- pixel rasters ---
    xs, ys, starts, Ns, shapes = [], [], [], [], []
    pos = 0
    for e in range(n_exp):
        if raster_width is None:
            w, h = exp_pix[e]
            n = w * h
            W = w
        else:
            n = int(exp_pix[e])
            W = raster_width
            h = -(-n // W)
            w = W
        idx = np.arange(n)
        x = (idx % W).astype(np.float32)
        y = (idx // W).astype(np.float32)
        npad = (-n) % PAD
        xs.append(np.concatenate([x, -np.ones(npad, np.float32)]))
        ys.append(np.concatenate([y, -np.ones(npad, np.float32)]))
        starts.append(pos)
        Ns.append(n + npad)
        shapes.append((w, h, n))
        pos += n + npad

    patch = SyntheticPatch()
    patch.build_patch(npix=pos, n_sources=n_sources, n_radii=n_radii, n_bands=n_bands, n_exp=n_exp)
    patch.xpix[:] = np.concatenate(xs)
    patch.ypix[:] = np.concatenate(ys)
    patch.exposure_start[:] = starts
    patch.exposure_N[:] = Ns
    patch.band_N[:] = exp_per_band
    patch.band_start[:] = np.concatenate([[0], np.cumsum(exp_per_band)[:-1]])
    patch.rad2[:] = radii ** 2
    patch.G[:] = 1.0
    patch.original_shapes = shapes

    # --- per-exposure linear astrometry: pixel = c_e + A_e (arcsec offset) ---
    A, cen = [], []
    for e in range(n_exp):
        w, h, _ = shapes[e]
        if perturb_wcs:
            M = _rot(rng.uniform(-0.05, 0.05)) @ np.array([[1.0, rng.uniform(-0.02, 0.02)], [0.0, 1.0]])
            dither = rng.uniform(-0.5, 0.5, 2)
        else:
            M, dither = np.eye(2), np.zeros(2)
        A.append(M / PIXSCALE)
        cen.append(np.array([(w - 1) / 2.0, (h - 1) / 2.0]) + dither)

    # --- sources, placed uniformly in the first exposure's area ---
    w0, h0, n0 = shapes[0]
    rows0 = -(-n0 // w0)
    scene = Scene()
    bandlist = ["b%d" % b for b in range(n_bands)]
    for s in range(n_sources):
        g = Galaxy(filternames=bandlist, splines=splines)
        sp = source_params(rng, n_bands)
        if "pix" in sp:
            px = np.asarray(sp["pix"], dtype=np.float64)
        else:
            px = np.array([rng.uniform(0, w0 - 1), rng.uniform(0, max(rows0 - 1, 1))])
        # arcsec offset in the tangent plane, then degrees (ra offset carries 1/cos dec)
        arcsec = np.linalg.solve(A[0], px - cen[0])
        dec = arcsec[1] / 3600.0
        cosd = np.cos(np.deg2rad(REF_COORD[1] + dec))
        ra = arcsec[0] / 3600.0 / cosd
        g.ra, g.dec = ra, dec
        g.flux[:] = sp["flux"]
        g.q, g.pa, g.sersic, g.rhalf = sp["q"], sp["pa"], sp["sersic"], sp["rhalf"]
        scene.sources.append(g)

    # --- PSFs: one mixture per band, replicated over radius bins (and, in
    # the packed metadata, over sources) ---
    psfs = [_psf_mixture(rng, n_psf, psf_anisotropic, psf_offsets) for _ in range(n_bands)]
    patch.n_psf_per_source[:] = n_radii * n_psf
    psf_blocks = []
    for e in range(n_exp):
        amps, pc, cov = psfs[band_of_exp[e]]
        one = np.zeros(n_radii * n_psf, dtype=psf_dtype)
        for r in range(n_radii):
            for i in range(n_psf):
                j = r * n_psf + i
                one[j] = (amps[i], pc[i, 0], pc[i, 1], cov[i, 0, 0], cov[i, 1, 1], cov[i, 0, 1], r)
        psf_blocks.append(one)

    patch.astrometry = (np.array(A), np.array(cen))
    patch.psf_blocks = psf_blocks
    patch.splines = splines
    patch.bandlist = bandlist
    patch.band_of_exp = band_of_exp
    patch.pack_meta(scene)
    return patch


def add_noise(patch, rng, sigma, model=None):
    """data = model + N(0, sigma_e^2) on real pixels, ierr = 1/sigma_e; pads stay 0."""
    sig = np.broadcast_to(np.asarray(sigma, dtype=np.float64), (patch.n_exp,))
    patch.sigma = np.array(sig)
    patch.data[:] = 0
    patch.ierr[:] = 0
    for e in range(patch.n_exp):
        s0, n = int(patch.exposure_start[e]), int(patch.original_shapes[e][2])
        sl = slice(s0, s0 + n)
        noise = rng.standard_normal(n) * sig[e]
        m = 0.0 if model is None else model[sl].astype(np.float64)
        patch.data[sl] = (m + noise).astype(np.float32)
        patch.ierr[sl] = np.float32(1.0 / sig[e])
    patch._dirty_data = True
    return patch


def _render_and_noise(patch, rng, sigma, render):
    model = None
    if render is not None:
        model = render(patch, patch.scene.get_proposal())
    return add_noise(patch, rng, sigma, model)


def _broad_source(rng, n_bands):
    return dict(flux=np.exp(rng.uniform(np.log(1.0), np.log(100.0), n_bands)),
                q=rng.uniform(0.3, 0.95), pa=rng.uniform(-np.pi / 2, np.pi / 2),
                sersic=rng.uniform(1.0, 5.0), rhalf=rng.uniform(0.05, 0.5))


def config_small(seed=1, render=None, size=64):
    """1 band, 1 exposure, one source near the centre of a 64x64 patch."""
    rng = np.random.default_rng(seed)
    c = (size - 1) / 2.0

    def one(rng, nb):
        return dict(flux=np.full(nb, 10.0), q=0.7, pa=0.4, sersic=2.0, rhalf=0.15,
                    pix=(c + rng.uniform(-2, 2), c + rng.uniform(-2, 2)))

    p = make_patch(rng, n_sources=1, exp_per_band=[1], exp_pix=[(size, size)], n_psf=3,
                   psf_anisotropic=False, psf_offsets=False, perturb_wcs=False,
                   source_params=one)
    return _render_and_noise(p, rng, 1.0, render)


def config_multiband(seed=2, render=None, n_sources=16, n_bands=5, exp_per_band=2,
                     size=150, n_psf=4):
    """5 bands x 2 exposures of 150x150 px, 16 sources."""
    rng = np.random.default_rng(seed)
    p = make_patch(rng, n_sources=n_sources, exp_per_band=[exp_per_band] * n_bands,
                   exp_pix=[(size, size)] * (exp_per_band * n_bands), n_psf=n_psf,
                   source_params=_broad_source)
    return _render_and_noise(p, rng, rng.uniform(0.5, 2.0, p.n_exp), render)


def config_limits(seed=3, render=None, n_sources=30, n_bands=8, exp_per_band=4, size=256,
                  n_psf=6):
    """30 sources, 8 bands x 4 exposures of 256x256 px, 6-Gaussian PSFs."""
    return config_multiband(seed=seed, render=render, n_sources=n_sources, n_bands=n_bands,
                            exp_per_band=exp_per_band, size=size, n_psf=n_psf)


def batched_shapes(seed=4, n_patches=512, max_sources=30, max_bands=8, max_exp=4,
                   min_pix=32 ** 2, max_pix=256 ** 2):
    """The per-patch shape draws of the batched workload (cheap; no pixels)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_patches):
        ns = int(rng.integers(1, max_sources + 1))
        nb = int(rng.integers(1, max_bands + 1))
        epb = [int(v) for v in rng.integers(1, max_exp + 1, nb)]
        pix = [int(v) for v in rng.integers(min_pix, max_pix + 1, sum(epb))]
        out.append(dict(n_sources=ns, exp_per_band=epb, exp_pix=pix, seed=int(rng.integers(2 ** 31))))
    return out


def config_batched(seed=4, render=None, n_patches=512, **kw):
    """512 uneven patches (see module docstring); returns a list of patches."""
    patches = []
    for sh in batched_shapes(seed=seed, n_patches=n_patches, **kw):
        rng = np.random.default_rng(sh["seed"])
        p = make_patch(rng, n_sources=sh["n_sources"], exp_per_band=sh["exp_per_band"],
                       exp_pix=sh["exp_pix"], n_psf=4, source_params=_broad_source,
                       raster_width=256)
        patches.append(_render_and_noise(p, rng, rng.uniform(0.5, 2.0, p.n_exp), render))
    return patches


def config_hmc(seed=5, render=None, n_patches=128, **kw):
    """Patches drawn like ``limits`` (the device-resident HMC workload)."""
    rng = np.random.default_rng(seed)
    return [config_limits(seed=int(rng.integers(2 ** 31)), render=render, **kw)
            for _ in range(n_patches)]


CONFIGS = {"small": config_small, "multiband": config_multiband, "limits": config_limits,
           "batched": config_batched, "hmc": config_hmc}
