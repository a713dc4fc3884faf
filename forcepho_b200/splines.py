"""Sersic mixture amplitudes A_i(sersic, rhalf) and their derivatives.

forcepho approximates a Sersic profile by Gaussians of fixed radii whose
amplitudes depend on (sersic, rhalf).  The amplitudes are tabulated on a
rectangular (sersic, rhalf) grid and interpolated with one scipy
``RectBivariateSpline`` per radius, exactly as ``Galaxy.initialize_splines``
and the ``amplitudes`` / ``damplitude_dsersic`` / ``damplitude_drh``
properties do (forcepho/sources.py:623-681).  The derivatives are the
spline's own partial derivatives (``dx=1`` for sersic, ``dy=1`` for rhalf).

The table is the reference's ``sersic_splinedata_large.h5``, converted once to
``data/sersic_splinedata_large.npz`` by ``data/convert_splinedata.py``.
"""

import os

import numpy as np
from scipy.interpolate import RectBivariateSpline

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DEFAULT_SPLINEDATA = os.path.join(DATA_DIR, "sersic_splinedata_large.npz")


def load_splinedata(path=DEFAULT_SPLINEDATA):
    """Return dict(amplitudes, nsersic, rh, radii) from the ``.npz`` table."""
    with np.load(path) as d:
        return {k: d[k].copy() for k in ("amplitudes", "nsersic", "rh", "radii")}


class SersicSplines:
    """One bicubic interpolating spline per mixture radius.

    Parameters
    ----------
    splinedata : str
        Path to the ``.npz`` amplitude table.
    spline_smoothing : float or None
        Passed to ``RectBivariateSpline`` as ``s`` (None means interpolation).
    """

    def __init__(self, splinedata=DEFAULT_SPLINEDATA, spline_smoothing=None):
        tab = load_splinedata(splinedata)
        n, r, A = tab["nsersic"], tab["rh"], tab["amplitudes"]
        self.radii = tab["radii"]
        ngrid, rgrid = np.unique(n), np.unique(r)
        nn, nr = len(ngrid), len(rgrid)
        # the table is stored sersic-major, rhalf-minor (checked here)
        if not (np.array_equal(n.reshape(nn, nr)[:, 0], ngrid)
                and np.array_equal(r.reshape(nn, nr)[0], rgrid)):
            raise ValueError("spline table is not on a sersic-major rectangular grid")
        kw = {} if spline_smoothing is None else {"s": spline_smoothing}
        self.splines = [RectBivariateSpline(ngrid, rgrid, A[:, i].reshape(nn, nr), **kw)
                        for i in range(A.shape[1])]
        self.sersic_range = (float(n.min()), float(n.max()))
        self.rh_range = (float(r.min()), float(r.max()))

    @property
    def n_gauss(self):
        return len(self.radii)

    def amplitudes(self, sersic, rhalf):
        return np.array([float(s(sersic, rhalf)[0, 0]) for s in self.splines])

    def damplitude_dsersic(self, sersic, rhalf):
        return np.array([float(s(sersic, rhalf, dx=1)[0, 0]) for s in self.splines])

    def damplitude_drh(self, sersic, rhalf):
        return np.array([float(s(sersic, rhalf, dy=1)[0, 0]) for s in self.splines])

    def tck(self):
        """Knots and coefficients of every spline: (tx, ty, c[n_radii, ...], kx, ky).

        All radii share the same knot vectors (same grid, interpolation), which
        is what a device-side evaluator needs."""
        tx = [s.get_knots()[0] for s in self.splines]
        ty = [s.get_knots()[1] for s in self.splines]
        for a, b in zip(tx[1:], ty[1:]):
            if not (np.array_equal(a, tx[0]) and np.array_equal(b, ty[0])):
                raise ValueError("splines do not share knots")
        c = np.stack([s.get_coeffs() for s in self.splines])
        kx, ky = self.splines[0].degrees
        return tx[0], ty[0], c, kx, ky


_cache = {}


def default_splines():
    """Process-wide SersicSplines of the default table (building them takes ~0.1 s)."""
    if "default" not in _cache:
        _cache["default"] = SersicSplines()
    return _cache["default"]
