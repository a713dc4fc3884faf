"""Galaxy sources and scenes: the producers of proposals.

Mirrors the parts of forcepho/sources.py that feed the likelihood kernel:

* ``Galaxy.set_params`` / ``get_param_vector`` (sources.py:559-605): a source's
  parameter vector is ``[flux_1 .. flux_nb, ra, dec, q, pa, sersic, rhalf]``;
* ``Galaxy.proposal`` (sources.py:607-621): pack one ``source_struct_dtype``
  record, with spline amplitudes and derivatives at (sersic, rhalf);
* ``Scene.set_all_source_params`` / ``get_all_source_params`` /
  ``get_proposal`` (sources.py:46-97).
"""

import numpy as np

from .splines import default_splines
from .structs import source_struct_dtype

__all__ = ["Galaxy", "Scene"]


class Galaxy:
    """A Sersic galaxy with per-band fluxes.

    ``q`` is sqrt(b/a) and ``pa`` the position angle in radians, as in the
    reference (sources.py:247-250); ``ra``/``dec`` are degree offsets from the
    patch reference coordinate.
    """

    SHAPE_COLS = ["ra", "dec", "q", "pa", "sersic", "rhalf"]
    npos, nshape = 2, 4

    def __init__(self, filternames=("band",), splines=None):
        self.filternames = list(filternames)
        self.flux = np.zeros(len(self.filternames))
        self.ra = self.dec = 0.0
        self.q, self.pa = 1.0, 0.0
        self.sersic, self.rhalf = 2.0, 0.1
        self.fixed = False
        self.splines = splines if splines is not None else default_splines()
        self.radii = self.splines.radii
        self.proposal_struct = np.zeros(1, dtype=source_struct_dtype)

    @property
    def n_bands(self):
        return len(self.filternames)

    @property
    def n_params(self):
        return self.n_bands + self.npos + self.nshape

    @property
    def n_gauss(self):
        return len(self.radii)

    def set_params(self, theta):
        theta = np.asarray(theta, dtype=np.float64)
        if len(theta) != self.n_params:
            raise ValueError("The length of the parameter vector is not appropriate for this source")
        nb = self.n_bands
        self.flux[:] = theta[:nb]
        self.ra, self.dec, self.q, self.pa, self.sersic, self.rhalf = theta[nb:nb + 6]

    def get_param_vector(self):
        return np.concatenate([self.flux, [self.ra, self.dec, self.q, self.pa,
                                           self.sersic, self.rhalf]])

    @property
    def amplitudes(self):
        return self.splines.amplitudes(self.sersic, self.rhalf)

    @property
    def damplitude_dsersic(self):
        return self.splines.damplitude_dsersic(self.sersic, self.rhalf)

    @property
    def damplitude_drh(self):
        return self.splines.damplitude_drh(self.sersic, self.rhalf)

    def proposal(self):
        p = self.proposal_struct
        p["fluxes"][0, :self.n_bands] = self.flux
        p["ra"], p["dec"] = self.ra, self.dec
        p["q"], p["pa"] = self.q, self.pa
        p["nsersic"], p["rh"] = self.sersic, self.rhalf
        p["mixture_amplitudes"][0, :self.n_gauss] = self.amplitudes
        p["damplitude_drh"][0, :self.n_gauss] = self.damplitude_drh
        p["damplitude_dnsersic"][0, :self.n_gauss] = self.damplitude_dsersic
        return p


class Scene:
    """An ordered collection of sources; maps the flat parameter vector."""

    def __init__(self, sources=()):
        self.sources = list(sources)

    def __len__(self):
        return len(self.sources)

    @property
    def active_sources(self):
        return [s for s in self.sources if not s.fixed]

    @property
    def n_active(self):
        return len(self.active_sources)

    def set_all_source_params(self, theta):
        start = 0
        for s in self.active_sources:
            s.set_params(theta[start:start + s.n_params])
            start += s.n_params

    def get_all_source_params(self, active=True):
        srcs = self.active_sources if active else self.sources
        return np.concatenate([s.get_param_vector() for s in srcs])

    def get_proposal(self, active=True):
        srcs = self.active_sources if active else [s for s in self.sources if s.fixed]
        return np.concatenate([s.proposal() for s in srcs])
