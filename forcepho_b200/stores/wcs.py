"""Gnomonic (TAN) world coordinate systems from FITS headers.

The reference takes every exposure's astrometry from ``astropy.wcs.WCS``
(forcepho/patches/pixel_patch.py:417, ``all_world2pix`` in
forcepho/patches/patch.py:340 and forcepho/region.py, ``pixel_scale_matrix``
in ``scale_at_sky``, forcepho/patches/patch.py:504-560).  astropy is not
installed here; ``TanWCS`` implements the part of it those calls use for the
headers forcepho's images carry: a celestial RA---TAN / DEC--TAN pair with a
linear CD (or PC x CDELT) matrix and no distortion terms, following the FITS
WCS papers (Greisen & Calabretta 2002; Calabretta & Greisen 2002, sections
2.3, 5.1.3): intermediate world coordinates (x, y) = CD (p - CRPIX) in degrees,
the zenithal gnomonic projection R_theta = (180/pi) cot(theta), and the
spherical rotation with the native pole at (CRVAL1, CRVAL2, LONPOLE = 180).
Pixel coordinates follow astropy's ``origin`` convention (0: the first pixel
is 0, 1: FITS's 1).
"""

import numpy as np

__all__ = ["TanWCS", "scale_at_sky"]

_R2D = 180.0 / np.pi


class TanWCS:
    """A TAN (gnomonic) celestial WCS without distortion."""

    def __init__(self, header):
        h = header
        c1, c2 = str(h.get("CTYPE1", "")), str(h.get("CTYPE2", ""))
        if not (c1.startswith("RA") and c1.endswith("-TAN") and c2.startswith("DEC") and c2.endswith("-TAN")):
            raise ValueError("only RA---TAN / DEC--TAN headers are supported (got %r, %r)" % (c1, c2))
        if any(k in h for k in ("A_ORDER", "B_ORDER", "PV1_1", "PV2_1", "PV2_2")):
            raise ValueError("distortion terms (SIP / PV) are not supported")
        self.crpix = np.array([float(h["CRPIX1"]), float(h["CRPIX2"])])
        self.crval = np.array([float(h["CRVAL1"]), float(h["CRVAL2"])])
        if "CD1_1" in h:
            cd = np.array([[float(h.get("CD1_1", 0.0)), float(h.get("CD1_2", 0.0))],
                           [float(h.get("CD2_1", 0.0)), float(h.get("CD2_2", 0.0))]])
        else:
            pc = np.array([[float(h.get("PC1_1", 1.0)), float(h.get("PC1_2", 0.0))],
                           [float(h.get("PC2_1", 0.0)), float(h.get("PC2_2", 1.0))]])
            cdelt = np.array([float(h.get("CDELT1", 1.0)), float(h.get("CDELT2", 1.0))])
            cd = cdelt[:, None] * pc
        self.cd = cd
        self.cd_inv = np.linalg.inv(cd)
        self.lonpole = float(h.get("LONPOLE", 180.0))
        self.has_distortion = False

    @property
    def pixel_scale_matrix(self):
        """Degrees per pixel (the CD matrix), as astropy's attribute of that name."""
        return self.cd

    def all_pix2world(self, x, y, origin):
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        p = np.stack([x + (1 - origin) - self.crpix[0], y + (1 - origin) - self.crpix[1]])
        X = self.cd[0, 0] * p[0] + self.cd[0, 1] * p[1]
        Y = self.cd[1, 0] * p[0] + self.cd[1, 1] * p[1]
        # native spherical coordinates of the gnomonic projection
        R = np.hypot(X, Y)
        phi = np.arctan2(X, -Y)
        theta = np.arctan2(_R2D, R)
        # native -> celestial, native pole at (alpha_p, delta_p), phi_p = LONPOLE
        a0, d0 = np.deg2rad(self.crval[0]), np.deg2rad(self.crval[1])
        dphi = phi - np.deg2rad(self.lonpole)
        st, ct = np.sin(theta), np.cos(theta)
        ra = a0 + np.arctan2(-ct * np.sin(dphi), st * np.cos(d0) - ct * np.sin(d0) * np.cos(dphi))
        dec = np.arcsin(np.clip(st * np.sin(d0) + ct * np.cos(d0) * np.cos(dphi), -1.0, 1.0))
        return np.mod(np.rad2deg(ra), 360.0), np.rad2deg(dec)

    def all_world2pix(self, ra, dec, origin):
        a = np.deg2rad(np.asarray(ra, np.float64))
        d = np.deg2rad(np.asarray(dec, np.float64))
        a0, d0 = np.deg2rad(self.crval[0]), np.deg2rad(self.crval[1])
        da = a - a0
        # the rotated unit vector (cos t cos(phi - phi_p), cos t sin(phi - phi_p), sin t):
        # theta from its components (an arcsin near the tangent point, where
        # theta -> 90 deg, would lose half the digits)
        u = np.sin(d) * np.cos(d0) - np.cos(d) * np.sin(d0) * np.cos(da)
        v = -np.cos(d) * np.sin(da)
        w = np.sin(d) * np.sin(d0) + np.cos(d) * np.cos(d0) * np.cos(da)
        phi = np.deg2rad(self.lonpole) + np.arctan2(v, u)
        R = _R2D * np.hypot(u, v) / w
        X, Y = R * np.sin(phi), -R * np.cos(phi)
        px = self.cd_inv[0, 0] * X + self.cd_inv[0, 1] * Y
        py = self.cd_inv[1, 0] * X + self.cd_inv[1, 1] * Y
        return px + self.crpix[0] - (1 - origin), py + self.crpix[1] - (1 - origin)


def scale_at_sky(sky, wcs):
    """Local linear astrometry at ``sky`` = (ra, dec) degrees, as the
    reference's ``scale_at_sky`` for a WCS without distortion
    (forcepho/patches/patch.py:504-560): D (pixels per arcsec, the inverse of
    3600 x the pixel scale matrix) and CW = 3600 D diag(cos dec, 1) (pixels per
    degree of (ra, dec)).  Returns (CW, D)."""
    W = np.eye(2)
    W[0, 0] = np.cos(np.deg2rad(sky[1]))
    D = np.linalg.inv(wcs.pixel_scale_matrix * 3600.0)
    CW = np.matmul(D * 3600.0, W)
    return CW, D
