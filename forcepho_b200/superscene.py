"""The catalog of every source in a survey field, and regions checked out of it.

Restates forcepho's parent-side scene bookkeeping (forcepho/superscene.py):
a master catalog (``sourcecat``) with per-source state columns, sky positions
mapped to *scene coordinates* (arcsec of longitude and latitude in the offset
frame centred on the catalog's median position) and a KD-tree over them.  A
region is *checked out* around a seed source: the sources that fit are marked
active, their neighbours fixed, and both become unavailable to later
checkouts until the region is *checked in* with new parameters.  Regions
checked out at the same time therefore never share an active source (a
fixed source, which is only subtracted, may serve several), which is what
lets many patches be evaluated in one batched launch, or on different GPUs,
without any exchange between them (``forcepho_b200.dispatcher``).

* ``SuperScene``        -- circular scenes: actives sorted by outer distance
  (distance + nscale rhalf) up to ``maxactive_per_patch`` and ``maxradius``
  (superscene.py:229-440);
* ``LinkedSuperScene``  -- scenes grown by friends-of-friends over the
  sources' radii of influence (superscene.py:495-748);
* prior-bound helpers ``make_bounds``, ``bounds_vectors``, ``check_bounds``,
  ``flux_bounds``, ``adjust_bounds``, and ``rectify_catalog``, ``convert_pa``
  (superscene.py:751-1050).

Differences from the reference, all where its code cannot run as written:
the sky-offset frame is a plain spherical rotation (astropy is not a
dependency); the random seed draw weights *valid* sources (the reference's
``exp_weight`` weights the invalid ones through ``~is_valid`` and uses the
removed ``np.float``, so its own random draw fails on a fresh scene); draws
use a seedable ``numpy.random.Generator``; ``convert_pa`` wraps angles into
[-pi/2, pi/2] as its docstring says (the reference's loop compares with
+pi/2 on both sides and, for the default even ``max_try``, returns its
input); a random draw with every source checked out gives no region instead
of normalising zero weights.  The state file is written with this package's
FITS writer.
"""

import json

import numpy as np
from scipy.linalg import block_diag
from scipy.spatial import cKDTree

from .sources import Galaxy
from .stores import fits as F
from .stores.region import CircularRegion

__all__ = ["REQUIRED_COLUMNS", "SuperScene", "LinkedSuperScene", "sky_to_offset", "sourcecat_dtype",
           "rectify_catalog", "convert_pa", "make_bounds", "bounds_vectors", "check_bounds", "flux_bounds",
           "adjust_bounds"]

REQUIRED_COLUMNS = ("ra", "dec", "rhalf", "source_index", "is_active", "is_valid", "n_iter", "n_patch")

ARCSEC_PER_RAD = 180.0 / np.pi * 3600.0


def sky_to_offset(ra, dec, ra0, dec0):
    """(lon, lat) in arcsec of (ra, dec) degrees in the offset frame whose
    origin is (ra0, dec0): the sphere rotated about the pole by -ra0, then
    about the new y axis by dec0, so that the origin lands on (1, 0, 0);
    longitude grows with RA and latitude with declination there."""
    a = np.deg2rad(np.asarray(ra, dtype=np.float64))
    d = np.deg2rad(np.asarray(dec, dtype=np.float64))
    a0, d0 = np.deg2rad(float(ra0)), np.deg2rad(float(dec0))
    cd = np.cos(d)
    x1, y1, z1 = cd * np.cos(a - a0), cd * np.sin(a - a0), np.sin(d)
    x2 = x1 * np.cos(d0) + z1 * np.sin(d0)
    z2 = z1 * np.cos(d0) - x1 * np.sin(d0)
    lon = np.arctan2(y1, x2)
    lat = np.arcsin(np.clip(z2, -1.0, 1.0))
    return lon * ARCSEC_PER_RAD, lat * ARCSEC_PER_RAD


def sourcecat_dtype(source_type=np.float64, bands=()):
    """The master catalog's row layout: state columns, the radius of
    influence, the shape columns and one flux column per band
    (superscene.py:751-764)."""
    dt = [(t, np.int32) for t in ("id", "source_index", "is_active", "is_valid", "n_iter", "n_patch")]
    dt += [("roi", np.float32)]
    dt += [(c, source_type) for c in Galaxy.SHAPE_COLS]
    dt += [(c, source_type) for c in bands]
    return np.dtype(dt)


class SuperScene:
    """All sources of a field, with regions checked out of and into it
    (superscene.py:36-492).

    Parameters
    ----------
    sourcecat : structured array with at least ``REQUIRED_COLUMNS``, the
        shape columns and one flux column per band (``sourcecat_dtype``).
        The scene keeps (and updates) this array.
    bands : the flux column names.
    target_niter, maxactive_fraction : stopping criteria (``undone``,
        ``sparse``).
    maxactive_per_patch, nscale, boundary_radius, maxradius, minradius :
        region geometry, arcsec (radii) and half-light radii (``nscale``).
    rng : ``numpy.random.Generator`` for the random seed draws.
    """

    sourcecat = None
    n_sources = 0

    def __init__(self, sourcecat=None, bands=None, statefile="superscene.fits", target_niter=200,
                 maxactive_fraction=0.1, maxactive_per_patch=20, nscale=3, boundary_radius=8., maxradius=6.,
                 minradius=1, bounds_kwargs=None, rng=None):
        self.statefilename = statefile
        self.bands = list(bands or [])
        self.shape_cols = list(Galaxy.SHAPE_COLS)
        self.rng = rng if rng is not None else np.random.default_rng()
        self.bounds_kwargs = dict(bounds_kwargs or {})
        if sourcecat is not None:
            self.ingest(sourcecat, **self.bounds_kwargs)
        self.n_active = 0
        self.n_fixed = 0
        self.maxactive_fraction = maxactive_fraction
        self.target_niter = target_niter
        self.maxradius = maxradius
        self.minradius = minradius
        self.maxactive = maxactive_per_patch
        self.boundary_radius = boundary_radius
        self.nscale = nscale

    def __enter__(self):
        return self

    def __exit__(self, extype, value, traceback):
        self.writeout()

    def writeout(self, filename=None):
        """The catalog as a FITS binary table, and the source/patch logs as
        JSON beside it (``*_log.json``)."""
        filename = filename or self.statefilename
        F.write_fits(filename, [({}, None), ({"EXTNAME": "SCENE"}, self.sourcecat)])
        with open(filename.replace(".fits", "_log.json"), "w") as f:
            json.dump(dict(sourcelog=self.sourcelog, patchlog=self.patchlog), f)

    # --- state ---
    @property
    def sparse(self):
        return self.n_sources > 0 and self.n_active * 1.0 / self.n_sources < self.maxactive_fraction

    @property
    def undone(self):
        return bool(np.any(np.abs(self.sourcecat["n_iter"]) < self.target_niter))

    @property
    def parameter_columns(self):
        return self.bands + self.shape_cols

    @property
    def cat_dtype(self):
        return self.sourcecat.dtype

    def ingest(self, sourcecat, **bounds_kwargs):
        """Take the catalog; build the KD-tree, the prior bounds and identity
        covariance matrices; start the logs."""
        self.set_catalog(sourcecat)
        self.kdt = cKDTree(self.scene_coordinates)
        self.bounds_catalog = make_bounds(self.sourcecat, self.bands, shapenames=self.shape_cols, **bounds_kwargs)
        n_param = len(self.parameter_columns)
        self.covariance_matrices = np.tile(np.eye(n_param), (self.n_sources, 1, 1))
        self.sourcelog = {}
        self.patchlog = []

    def check_bounds(self):
        check_bounds(self.sourcecat, self.bounds_catalog)

    def set_catalog(self, sourcecat):
        missing = [c for c in tuple(REQUIRED_COLUMNS) + tuple(self.bands) if c not in sourcecat.dtype.names]
        if missing:
            raise ValueError("required columns not in the catalog: %s" % ", ".join(missing))
        self.sourcecat = sourcecat
        self.n_sources = len(sourcecat)
        self.sourcecat["source_index"][:] = np.arange(self.n_sources)
        self.sourcecat["is_valid"][:] = True
        self.sourcecat["is_active"][:] = False
        self.original = sourcecat.copy()
        for attr in ("_scene_center", "_scene_coordinates"):
            self.__dict__.pop(attr, None)

    # --- coordinates ---
    @property
    def scene_center(self):
        """(ra, dec) degrees of the scene frame's origin: the catalog's median position."""
        if "_scene_center" not in self.__dict__:
            if self.n_sources == 0:
                self._scene_center = (0.0, 0.0)
            else:
                self._scene_center = (float(np.median(self.sourcecat["ra"])),
                                      float(np.median(self.sourcecat["dec"])))
        return self._scene_center

    def sky_to_scene(self, ra, dec):
        """Scene coordinates (lon, lat), arcsec, of (ra, dec) degrees."""
        return sky_to_offset(ra, dec, *self.scene_center)

    @property
    def scene_coordinates(self):
        """[n_sources, 2] scene coordinates of the catalog's original positions."""
        if "_scene_coordinates" not in self.__dict__:
            x, y = self.sky_to_scene(self.sourcecat["ra"], self.sourcecat["dec"])
            self._scene_coordinates = np.array([x, y]).T
        return self._scene_coordinates

    # --- checkout / checkin ---
    def checkout_region(self, seed_index=-1):
        """A circular region around a seed source (drawn when ``seed_index`` <
        0) and copies of its active and fixed catalog rows; those sources are
        marked unavailable.  Returns (center, None, None) when the region
        would contain an active source."""
        seed = self.draw_center(seed_index=seed_index)
        if seed is None:
            return None, None, None
        cra, cdec = seed
        center = self.sky_to_scene(cra, cdec)
        radius, active_inds, fixed_inds = self.get_circular_scene(center)
        if radius is None:
            return center, None, None
        region = CircularRegion(cra, cdec, radius / 3600.)
        self.sourcecat["is_active"][active_inds] = True
        self.sourcecat["is_valid"][active_inds] = False
        self.sourcecat["is_valid"][fixed_inds] = False
        self.n_active += len(active_inds)
        self.n_fixed += len(fixed_inds)
        return region, self.sourcecat[active_inds], self.sourcecat[fixed_inds]

    def checkin_region(self, active, fixed=None, niter=1, block_covs=None, new_bounds=None, taskID=None,
                       flush=False):
        """Write the active sources' new parameters back, make the region's
        sources available again and count the iterations; optionally update
        their bounds and covariance blocks, log the task, flush to disk."""
        active_inds = np.asarray(active["source_index"]).astype(int)
        fixed_inds = np.asarray(fixed["source_index"]).astype(int) if fixed is not None else np.zeros(0, int)
        for c in self.parameter_columns:
            self.sourcecat[c][active_inds] = active[c]
        self.sourcecat["n_iter"][active_inds] += niter
        self.sourcecat["is_active"][active_inds] = False
        self.sourcecat["n_patch"][active_inds] += int(niter > 0)
        self.sourcecat["is_valid"][active_inds] = True
        self.sourcecat["is_valid"][fixed_inds] = True
        self.n_active -= len(active_inds)
        self.n_fixed -= len(fixed_inds)
        if new_bounds is not None:
            self.bounds_catalog[active_inds] = new_bounds[:]
        if block_covs is not None:
            self.covariance_matrices[active_inds] = block_covs
        if taskID is not None:
            pid = str(taskID)
            for k in active_inds:
                self.sourcelog.setdefault(int(k), []).append(pid)
            self.patchlog.append(pid)
        if flush:
            self.writeout()

    def bounds_and_covs(self, sourceIDs):
        """Bounds rows and the block-diagonal covariance of the given sources."""
        covs = self.covariance_matrices[sourceIDs]
        return self.bounds_catalog[sourceIDs], block_diag(*covs)

    def reset(self):
        self.sourcecat["is_valid"][:] = True
        self.sourcecat["is_active"][:] = False
        self.sourcecat["n_iter"][:] = 0
        self.sourcecat["n_patch"][:] = 0
        self.n_active = 0
        self.n_fixed = 0

    def get_circular_scene(self, center):
        """(radius arcsec, active indices, fixed indices) of the circular scene
        at ``center`` (scene coordinates), or (None, None, None) if a source
        within ``boundary_radius`` is active.

        Candidates are the sources within ``boundary_radius``, ordered by their
        outer distance (distance + nscale rhalf).  Those with outer distance
        below ``maxradius`` become active, at most ``maxactive``; the radius is
        the largest active outer distance (at least ``minradius``); fixed are
        the remaining candidates whose inner distance (distance - nscale
        rhalf) is within the radius, at most ``maxactive``, and at least the
        nearest one."""
        kinds = np.array(self.kdt.query_ball_point(center, self.boundary_radius), dtype=int)
        if np.any(self.sourcecat[kinds]["is_active"]):
            return None, None, None
        rhalf = self.sourcecat[kinds]["rhalf"]
        d = self.scene_coordinates[kinds] - np.asarray(center, dtype=np.float64)
        distance = np.hypot(*d.T)
        outer = distance + self.nscale * rhalf
        inner = distance - self.nscale * rhalf
        order = np.argsort(outer)
        n_active = min(self.maxactive, int((outer < self.maxradius).sum()))
        if n_active == 0:
            return None, None, None
        active_inds = order[:n_active]
        others = order[n_active:]
        radius = max(self.minradius, outer[active_inds].max())
        fixed_inds = others[inner[others] < radius][:min(self.maxactive, len(others))]
        if len(fixed_inds) == 0:
            fixed_inds = others[:1]
        return radius, kinds[active_inds], kinds[fixed_inds]

    def draw_seed(self):
        """A random source index drawn with ``seed_weight`` probabilities, or
        -1 when no source has weight (every source checked out)."""
        w = self.seed_weight()
        if self.n_sources == 0 or not np.all(np.isfinite(w)) or w.sum() <= 0:
            return -1
        return int(self.rng.choice(self.n_sources, p=w))

    def draw_center(self, seed_index=-1):
        """(ra, dec) of the seed source: ``seed_index`` if >= 0, else a random
        draw (``draw_seed``); None when there is nothing to draw."""
        k = seed_index if seed_index >= 0 else self.draw_seed()
        if k < 0:
            return None
        seed = self.sourcecat[k]
        return seed["ra"], seed["dec"]

    def seed_weight(self):
        return self.exp_weight()

    def exp_weight(self):
        """Valid sources, down-weighted by exp(-(n_iter - mean n_iter) / 20)."""
        w = (self.sourcecat["is_valid"] != 0).astype(np.float64)
        n = np.abs(self.sourcecat["n_iter"]).astype(np.float64)
        if len(n):
            w *= np.exp((n.mean() - n) / 20.0)
        t = w.sum()
        return w / t if t > 0 else w

    def sigmoid_weight(self):
        """Inactive sources, weighted by a sigmoid of 1 - n_iter / target_niter."""
        w = (self.sourcecat["is_active"] == 0).astype(np.float64)
        a, b = 20., -1.0
        x = a * (1 - self.sourcecat["n_iter"] / self.target_niter) + b
        w *= 1 / (1 + np.exp(-x))
        t = w.sum()
        return w / t if t > 0 else w


class LinkedSuperScene(SuperScene):
    """Scenes grown by friends-of-friends: two sources are linked when their
    distance is below the sum of their radii of influence (``roi``, default
    rhalf); a scene adds whole linked groups in order of distance from the
    seed (superscene.py:495-748).

    Extra parameters: ``buffer`` (arcsec added to the enclosing radius),
    ``roi`` (arcsec per source), ``strict`` (leave slots empty rather than
    add part of a group, unless the scene is still empty)."""

    def __init__(self, *args, buffer=0.3, roi=None, strict=False, **kwargs):
        super().__init__(*args, **kwargs)
        self.buffer = buffer
        self.strict = strict
        self.roi = np.asarray(self.sourcecat["rhalf"] if roi is None else roi, dtype=np.float64)

    def grow_source(self, index):
        """Indices of every source linked to ``index`` (itself first), in the
        order a breadth-first walk over the links reaches them."""
        members, seen = [], set()
        seeds = [int(index)]
        while seeds:
            members += seeds
            seen.update(seeds)
            leaves, pending = [], set()
            for s in seeds:
                for b in self.find_overlaps(self.scene_coordinates[s], self.roi[s], seed_index=s).tolist():
                    if b not in pending:
                        pending.add(b)
                        leaves.append(b)
            seeds = [b for b in leaves if b not in seen]
        return members

    def grow_scene(self, seed_index, max_fixed=None):
        """(region, active indices, fixed indices) of the scene grown from the
        seed; ((ra, dec) of the seed, None, None) if a source within
        ``boundary_radius`` is active.  Groups are added nearest first until
        ``maxactive`` would be exceeded; the region is centred on the mean
        position of the actives, its radius encloses their radii of influence
        plus ``buffer``; fixed are the other sources overlapping 1.2 times it,
        nearest first, at most ``max_fixed`` (default ``maxactive``)."""
        seed = self.original[seed_index]
        candidates = self.find_overlaps(self.scene_coordinates[seed_index], self.boundary_radius, sort=True)
        if np.any(self.sourcecat[candidates]["is_active"]):
            return (seed["ra"], seed["dec"]), None, None
        active_inds = []
        for s in candidates.tolist():
            if s in active_inds:
                continue
            n_avail = self.maxactive - len(active_inds)
            to_add = self.grow_source(s)
            if len(to_add) > n_avail:
                if (not self.strict) or len(active_inds) == 0:
                    active_inds += to_add[:n_avail]
                break
            active_inds += to_add
        active = self.sourcecat[active_inds]
        cra, cdec = np.mean(active["ra"]), np.mean(active["dec"])
        center = np.array(self.sky_to_scene(cra, cdec))
        d = self.scene_coordinates[active_inds] - center
        radius = max(self.minradius, np.max(np.hypot(*d.T) + self.roi[active_inds] + self.buffer))
        region = CircularRegion(cra, cdec, radius / 3600.)
        max_fixed = self.maxactive if max_fixed is None else max_fixed
        inregion = self.find_overlaps(center, 1.2 * radius, sort=True)
        taken = set(active_inds)
        fixed_inds = [i for i in inregion.tolist() if i not in taken][:max_fixed]
        return region, active_inds, fixed_inds

    def checkout_region(self, seed_index=-1, max_fixed=None):
        """(region, active rows, fixed rows or None) of the scene grown from a
        seed (drawn when ``seed_index`` < 0), its sources marked unavailable;
        ((seed position, seed_index), None, None) when the seed's
        neighbourhood holds an active source."""
        if seed_index < 0:
            seed_index = self.draw_seed()
            if seed_index < 0:
                return (None, -1), None, None
        region, active_inds, fixed_inds = self.grow_scene(seed_index, max_fixed)
        if active_inds is None:
            return (region, seed_index), None, None
        fixed = self.sourcecat[fixed_inds] if len(fixed_inds) else None
        self.sourcecat["is_active"][active_inds] = True
        self.sourcecat["is_valid"][active_inds] = False
        self.sourcecat["is_valid"][fixed_inds] = False
        self.n_active += len(active_inds)
        self.n_fixed += len(fixed_inds)
        return region, self.sourcecat[active_inds], fixed

    def find_overlaps(self, center, radius, seed_index=-1, sort=False):
        """Indices of the sources k with |x_k - center| < radius + roi_k,
        excluding ``seed_index``; with ``sort``, in increasing order of
        |x_k - center| / (radius + roi_k)."""
        kinds = np.array(self.kdt.query_ball_point(center, radius + self.boundary_radius), dtype=int)
        d = self.scene_coordinates[kinds] - np.asarray(center, dtype=np.float64)
        metric = np.hypot(*d.T) / (radius + self.roi[kinds])
        overlaps = (metric < 1) & (metric >= 0) & (kinds != seed_index)
        order = np.argsort(metric[overlaps]) if sort else slice(None)
        return kinds[overlaps][order]

    def overlap_circle(self, ra, dec, radius):
        """Catalog rows of the sources whose roi overlaps the circle (radius in
        arcsec) around (ra, dec) degrees."""
        return self.sourcecat[self.find_overlaps(np.array(self.sky_to_scene(ra, dec)), radius)]

    def make_group_catalog(self):
        """The friends-of-friends group number of every source (from 0, in
        order of each group's lowest index)."""
        group = np.zeros(self.n_sources) - 1
        g = 0
        for i in range(self.n_sources):
            if group[i] >= 0:
                continue
            group[self.grow_source(i)] = g
            g += 1
        return group


# --- catalogs and prior bounds ---------------------------------------------
def _first_table(path):
    hdus = F.read_fits(path)
    for h in hdus:
        if h.data is not None and getattr(h.data, "dtype", None) is not None and h.data.dtype.names:
            return h.data, hdus[0].header
    raise ValueError("%s holds no binary table" % path)


def rectify_catalog(sourcecatfile, rhalf_range=(0.051, 0.29), sqrtq_range=(0.2, 0.99), sersic_range=(1.01, 4.99),
                    pa_range=(-2.0, 2.0), rotate=False, reverse=False, shapenames=tuple(Galaxy.SHAPE_COLS)):
    """(master catalog, bands, header) from a FITS source catalog (path, or a
    (table, header) pair) whose header lists its flux columns in FILTERS:
    columns copied into ``sourcecat_dtype`` rows (checked finite), shape
    parameters clipped to the given ranges, PA optionally rotated by +90
    degrees within [-pi/2, pi/2] and/or reversed (superscene.py:767-802)."""
    cat, header = _first_table(sourcecatfile) if isinstance(sourcecatfile, str) else sourcecatfile
    bands = [b.strip() for b in str(header["FILTERS"]).split(",")]
    for c in list(bands) + list(shapenames):
        if c not in cat.dtype.names:
            raise ValueError("'%s' column not in input catalog" % c)
    sourcecat = np.zeros(len(cat), dtype=sourcecat_dtype(bands=bands))
    sourcecat["source_index"][:] = np.arange(len(cat))
    for f in cat.dtype.names:
        if f in sourcecat.dtype.names:
            if not np.all(np.isfinite(cat[f][:])):
                raise ValueError("non-finite value in the '%s' column of the input catalog" % f)
            sourcecat[f][:] = cat[f][:]
    sourcecat["rhalf"][:] = np.clip(sourcecat["rhalf"], *rhalf_range)
    sourcecat["q"][:] = np.clip(sourcecat["q"], *sqrtq_range)
    sourcecat["sersic"][:] = np.clip(sourcecat["sersic"], *sersic_range)
    sourcecat["pa"][:] = np.clip(sourcecat["pa"], *pa_range)
    if rotate:
        p = sourcecat["pa"] > 0
        sourcecat["pa"] += np.pi / 2. - p * np.pi
    if reverse:
        sourcecat["pa"] *= -1.0
    return sourcecat, bands, header


def convert_pa(pa_in, from_deg=False, rotate=False, reverse=False, max_try=4):
    """Position angles in radians wrapped into [-pi/2, pi/2] (by whole turns
    of pi, at most ``max_try`` of them), optionally rotated by +90 degrees
    (staying in the interval) and/or reversed (superscene.py:1005-1040)."""
    pa = np.deg2rad(pa_in) if from_deg else np.array(pa_in, dtype=np.float64, copy=True)
    for _ in range(max_try):
        hi, lo = pa > np.pi / 2, pa < -np.pi / 2
        if not (hi.any() or lo.any()):
            break
        pa[hi] -= np.pi
        pa[lo] += np.pi
    if rotate:
        p = pa > 0
        pa += np.pi / 2. - p * np.pi
    if reverse:
        pa *= -1.0
    return pa


def make_bounds(active, filternames, shapenames=tuple(Galaxy.SHAPE_COLS), unccat=None, n_sig_flux=5., dpos=None,
                n_pix=2, pixscale=0.03, sqrtq_range=(0.4, 1.0), pa_range=(-0.6 * np.pi, 0.6 * np.pi),
                rhalf_range=(0.03, 0.3), sersic_range=(1., 5.)):
    """Per-source (lower, upper) prior bounds as a structured array, one
    (2,)-field per parameter (superscene.py:805-881): fixed ranges for q, pa,
    sersic and rhalf; ra/dec within ``dpos`` arcsec (default ``n_pix``
    pixels) of the catalog position; fluxes within ``n_sig_flux`` of the
    uncertainty catalog (floored at 5 % of the flux), else ``flux_bounds``.
    ``source_index`` is left 0, as the reference leaves it."""
    pm1 = np.array([-1., 1.])
    dpos = np.ones(2) * n_pix * pixscale if dpos is None else np.asarray(dpos, dtype=np.float64)
    dra = dpos[0] / 3600. / np.cos(np.deg2rad(active["dec"]))
    ddec = np.array([dpos[1] / 3600.])
    cols = list(filternames) + list(shapenames)
    bcat = np.zeros(len(active), dtype=np.dtype([("source_index", np.int32)] + [(c, np.float64, (2,)) for c in cols]))
    bcat["q"] = sqrtq_range
    bcat["pa"] = pa_range
    bcat["sersic"] = sersic_range
    bcat["rhalf"] = rhalf_range
    bcat["ra"] = active["ra"][:, None] + pm1[None, :] * dra[:, None]
    bcat["dec"] = active["dec"][:, None] + pm1[None, :] * ddec[:, None]
    for b in filternames:
        if unccat is not None:
            sigma = np.maximum(unccat[b], np.abs(0.05 * active[b]))
            lo, hi = active[b] + pm1[:, None] * n_sig_flux * sigma[None, :]
        else:
            lo, hi = flux_bounds(active[b], n_sig_flux)
        bcat[b][:, 0] = lo
        bcat[b][:, 1] = hi
    return bcat


def bounds_vectors(bounds_cat, filternames, shapenames=tuple(Galaxy.SHAPE_COLS), reference_coordinates=(0., 0.)):
    """Flat (lower, upper) vectors over sources, each source's fluxes then
    shape parameters, ra/dec relative to ``reference_coordinates``
    (superscene.py:884-899)."""
    bcat = bounds_cat.copy()
    bcat["ra"] -= reference_coordinates[0]
    bcat["dec"] -= reference_coordinates[1]
    cols = list(filternames) + list(shapenames)
    lower = np.array([[row[c][0] for c in cols] for row in bcat]).ravel()
    upper = np.array([[row[c][1] for c in cols] for row in bcat]).ravel()
    return lower, upper


def check_bounds(sourcecat, boundscat):
    """Raise AssertionError naming the column if any value is not strictly
    inside its (lower, upper) bound (superscene.py:902-919)."""
    for c in boundscat.dtype.names:
        b = boundscat[c][:]
        if b.shape[-1] != 2 or b.shape == (2,):
            continue
        if not np.all(sourcecat[c] > b[:, 0]):
            raise AssertionError("An input value is below lower bound in column '%s'" % c)
        if not np.all(sourcecat[c] < b[:, 1]):
            raise AssertionError("An input value is above bound in column '%s'" % c)


def flux_bounds(flux, unc1, snr_max=10, precisions=None):
    """(lower, upper) flux bounds (superscene.py:922-965).  With a precision
    matrix: flux -+ unc1 sigma, sigma from its pseudo-inverse floored at
    flux / snr_max, the upper bound at least unc1 sigma.  Without: a
    half-width of |flux| / (sqrt|flux| / unc1), widened to at least
    (unc1/2)^2 on each side of faint fluxes; non-finite bounds replaced."""
    flux = np.asarray(flux, dtype=np.float64)
    if flux.size == 0:
        return flux.copy(), flux.copy()
    if precisions is not None:
        sigma = np.maximum(np.sqrt(np.diag(np.linalg.pinv(precisions))), flux / snr_max)
        lo = flux - unc1 * sigma
        hi = np.maximum(flux + unc1 * sigma, unc1 * sigma)
        return lo, hi
    with np.errstate(divide="ignore", invalid="ignore"):
        snr = np.sqrt(np.abs(flux)) / unc1
        noise = np.abs(flux) / snr
    fmin = (unc1 / 2.) ** 2
    lo, hi = flux - noise, flux + noise
    faint = flux <= fmin
    lo[faint] = np.minimum(lo[faint], -fmin)
    lo[~np.isfinite(lo)] = 0
    hi = np.maximum(hi, fmin)
    hi[~np.isfinite(hi)] = np.nanmax(hi)
    return lo, hi


def adjust_bounds(sceneDB, bands, config, active=None, eps=0.001, minflux=None, maxfluxfactor=None):
    """Widen the flux bounds: lower bounds at most ``minflux``, upper bounds at
    least ``maxfluxfactor`` times the catalog flux; clip ``active``'s fluxes
    to eps inside the bounds; check the scene's bounds (superscene.py:968-1002).
    ``sceneDB`` is a scene, or a bounds array with ``active`` its catalog.
    The reference reads a ``source_catalog`` attribute that scenes do not
    have and clips to (lower + eps, lower - eps); this clips to
    (lower + eps, upper - eps)."""
    if isinstance(sceneDB, np.ndarray):
        bcat, scat = sceneDB, active
    else:
        bcat, scat = sceneDB.bounds_catalog, sceneDB.sourcecat
    minflux = getattr(config, "minflux", None) if minflux is None else minflux
    maxfluxfactor = getattr(config, "maxfluxfactor", 0) if maxfluxfactor is None else maxfluxfactor
    if minflux is not None:
        for b in bands:
            bcat[b][:, 0] = np.minimum(bcat[b][:, 0], minflux)
    if maxfluxfactor and maxfluxfactor > 0:
        for b in bands:
            bcat[b][:, 1] = np.maximum(bcat[b][:, 1], scat[b] * maxfluxfactor)
    if active is not None:
        for b in bands:
            active[b][:] = np.clip(active[b][:], bcat[b][:, 0] + eps, bcat[b][:, 1] - eps)
    if not isinstance(sceneDB, np.ndarray):
        sceneDB.check_bounds()
    return sceneDB
