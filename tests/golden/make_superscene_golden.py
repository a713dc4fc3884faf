"""Golden checkouts of forcepho's own SuperScene / LinkedSuperScene code.

Imports the reference's forcepho/superscene.py (and its forcepho.region,
forcepho.sources) from a reference checkout without running the package's
__init__, with two stand-ins for astropy, which is not installed:
``SkyCoord.transform_to(center.skyoffset_frame())`` as an explicit rotation
matrix (the offset frame's definition), and an empty ``astropy.io.fits``.
Everything else that runs -- the KD-tree queries, the ordering of candidates,
the radii, the active/fixed selection, friends-of-friends growth, checkin
bookkeeping and the bounds helpers -- is the reference's code.  Seeds are
given explicitly (the reference's random seed draw cannot run: see
forcepho_b200/superscene.py).

    python tests/golden/make_superscene_golden.py [REFERENCE_ROOT]

writes tests/golden/superscene_golden.json.
"""

import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def _rotation(ra0, dec0):
    a0, d0 = np.deg2rad(ra0), np.deg2rad(dec0)
    rz = np.array([[np.cos(a0), np.sin(a0), 0.], [-np.sin(a0), np.cos(a0), 0.], [0., 0., 1.]])
    ry = np.array([[np.cos(d0), 0., np.sin(d0)], [0., 1., 0.], [-np.sin(d0), 0., np.cos(d0)]])
    return ry @ rz


class _Angle:
    def __init__(self, rad):
        self.arcsec = np.degrees(rad) * 3600.0


class _Frame:
    def __init__(self, ra0, dec0):
        self.m = _rotation(ra0, dec0)


class _SkyCoord:
    def __init__(self, ra, dec, unit="deg"):
        self.ra, self.dec = np.asarray(ra, np.float64), np.asarray(dec, np.float64)

    def skyoffset_frame(self):
        return _Frame(float(self.ra), float(self.dec))

    def transform_to(self, frame):
        a, d = np.deg2rad(self.ra), np.deg2rad(self.dec)
        v = np.stack([np.cos(d) * np.cos(a), np.cos(d) * np.sin(a), np.sin(d)])
        w = np.tensordot(frame.m, v, axes=1)
        out = types.SimpleNamespace()
        out.lon = _Angle(np.arctan2(w[1], w[0]))
        out.lat = _Angle(np.arcsin(np.clip(w[2], -1, 1)))
        return out


def import_reference(root):
    pkg = types.ModuleType("forcepho")
    pkg.__path__ = [os.path.join(root, "forcepho")]
    sys.modules["forcepho"] = pkg
    astropy = types.ModuleType("astropy")
    io = types.ModuleType("astropy.io")
    fits = types.ModuleType("astropy.io.fits")
    coords = types.ModuleType("astropy.coordinates")
    coords.SkyCoord = _SkyCoord
    astropy.io, io.fits, astropy.coordinates = io, fits, coords
    sys.modules.update({"astropy": astropy, "astropy.io": io, "astropy.io.fits": fits,
                        "astropy.coordinates": coords})
    import forcepho.superscene as SS
    return SS


def catalog(SS, seed=20261204, n=400, bands=("F115W", "F200W", "F444W")):
    """Seeded field: 40 clumps of 1-20 sources plus uniform field sources,
    about 90 arcsec across around (53.1, -27.8)."""
    rng = np.random.default_rng(seed)
    ra0, dec0 = 53.1, -27.8
    cen = rng.uniform(-45, 45, (40, 2))
    pos = []
    while len(pos) < n:
        if rng.uniform() < 0.7:
            c = cen[rng.integers(40)]
            pos.append(c + rng.normal(0, 0.6, 2))
        else:
            pos.append(rng.uniform(-45, 45, 2))
    pos = np.array(pos[:n])
    cat = np.zeros(n, dtype=SS.sourcecat_dtype(bands=list(bands)))
    cat["id"] = np.arange(n) + 1000
    cat["ra"] = ra0 + pos[:, 0] / 3600. / np.cos(np.deg2rad(dec0))
    cat["dec"] = dec0 + pos[:, 1] / 3600.
    cat["rhalf"] = rng.uniform(0.05, 0.3, n)
    cat["roi"] = cat["rhalf"] * 3
    cat["q"] = rng.uniform(0.4, 0.95, n)
    cat["pa"] = rng.uniform(-1.5, 1.5, n)
    cat["sersic"] = rng.uniform(1.2, 4.5, n)
    for b in bands:
        cat[b] = np.exp(rng.uniform(np.log(0.5), np.log(200), n))
    return cat, list(bands)


SEEDS = [0, 7, 19, 33, 7, 58, 101, 150, 151, 222, 305, 399, 12, 64]


def circular(SS, cat, bands):
    sc = SS.SuperScene(sourcecat=cat.copy(), bands=bands, maxactive_per_patch=15, maxradius=6.,
                       boundary_radius=8., nscale=3, minradius=1)
    out = {"scene_coordinates": sc.scene_coordinates.tolist(), "checkouts": []}
    held = []
    for k, s in enumerate(SEEDS):
        region, active, fixed = sc.checkout_region(seed_index=s)
        rec = {"seed": s, "ok": active is not None}
        if active is not None:
            rec.update(ra=region.ra, dec=region.dec, radius=region.radius,
                       active=active["source_index"].tolist(), fixed=fixed["source_index"].tolist())
            held.append((active, fixed))
        out["checkouts"].append(rec)
        if k % 4 == 3 and held:             # check one region back in, with new parameters
            a, f = held.pop(0)
            a = a.copy()
            a["q"] = np.clip(a["q"] * 1.01, 0, 0.99)
            a[bands[0]] *= 1.5
            sc.checkin_region(a, f, niter=3, taskID=k)
    out["state"] = {c: sc.sourcecat[c].tolist() for c in ("is_active", "is_valid", "n_iter", "n_patch", "q",
                                                           bands[0])}
    out["n_active"], out["n_fixed"] = sc.n_active, sc.n_fixed
    bnd, cov = sc.bounds_and_covs(np.array([3, 8, 9]))
    out["bounds_and_covs_shape"] = list(cov.shape)
    return out


def linked(SS, cat, bands, strict):
    sc = SS.LinkedSuperScene(sourcecat=cat.copy(), bands=bands, maxactive_per_patch=15, maxradius=6.,
                             boundary_radius=8., nscale=3, minradius=1, buffer=0.3, roi=cat["roi"], strict=strict)
    out = {"grow": {str(s): sc.grow_source(s) for s in (0, 7, 19, 33, 150)},
           "groups": sc.make_group_catalog().tolist(), "checkouts": []}
    held = []
    for k, s in enumerate(SEEDS):
        region, active, fixed = sc.checkout_region(seed_index=s)
        rec = {"seed": s, "ok": active is not None}
        if active is not None:
            rec.update(ra=float(region.ra), dec=float(region.dec), radius=float(region.radius),
                       active=active["source_index"].tolist(),
                       fixed=[] if fixed is None else fixed["source_index"].tolist())
            held.append((active, fixed))
        out["checkouts"].append(rec)
        if k % 4 == 3 and held:
            a, f = held.pop(0)
            sc.checkin_region(a, f, niter=1)
    out["state"] = {c: sc.sourcecat[c].tolist() for c in ("is_active", "is_valid", "n_iter", "n_patch")}
    out["overlap_circle"] = sc.overlap_circle(53.1, -27.8, 2.0)["source_index"].tolist()
    return out


def bounds(SS, cat, bands):
    unc = np.zeros(len(cat), dtype=[(b, np.float64) for b in bands])
    rng = np.random.default_rng(5)
    for b in bands:
        unc[b] = np.abs(cat[b]) * rng.uniform(0.01, 0.2, len(cat))
    plain = SS.make_bounds(cat, bands)
    withunc = SS.make_bounds(cat, bands, unccat=unc, dpos=np.array([0.1, 0.05]))
    lo, hi = SS.bounds_vectors(plain[:5], bands, reference_coordinates=[53.1, -27.8])
    prec = np.diag(1.0 / np.linspace(0.5, 3.0, 6) ** 2)
    prec[0, 1] = prec[1, 0] = 0.1
    fl = np.array([-3.0, 0.01, 0.5, 2.0, 30.0, 400.0])
    return {"plain": {c: plain[c].tolist() for c in plain.dtype.names},
            "withunc": {c: withunc[c].tolist() for c in withunc.dtype.names},
            "unc": {b: unc[b].tolist() for b in bands},
            "vectors": [lo.tolist(), hi.tolist()],
            "flux_bounds": [x.tolist() for x in SS.flux_bounds(fl.copy(), 5.0)],
            "flux_bounds_prec": [x.tolist() for x in SS.flux_bounds(fl.copy(), 5.0, precisions=prec)],
            "flux_in": fl.tolist(), "prec": prec.tolist()}


def main():
    from oracle import oracle as O
    root = sys.argv[1] if len(sys.argv) > 1 else O.reference_root()
    SS = import_reference(root)
    cat, bands = catalog(SS)
    gold = {"bands": bands, "catalog": {c: cat[c].tolist() for c in cat.dtype.names},
            "circular": circular(SS, cat, bands), "linked": linked(SS, cat, bands, False),
            "linked_strict": linked(SS, cat, bands, True), "bounds": bounds(SS, cat, bands)}
    path = os.path.join(HERE, "superscene_golden.json")
    with open(path, "w") as f:
        json.dump(gold, f, default=lambda o: o.item())
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
