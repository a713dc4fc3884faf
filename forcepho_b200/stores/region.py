"""Sky regions that select a patch's pixels.

Restates the reference's ``CircularRegion`` and ``RectangularRegion``
(forcepho/region.py): a region in celestial coordinates, a bounding box used
to find the exposures that overlap it, and ``contains``: given the pixel
corners of an exposure and its WCS, the indices of the (super-)pixels with at
least one corner inside the region.
"""

import numpy as np

__all__ = ["CircularRegion", "RectangularRegion"]


class CircularRegion:
    """A circle of ``radius`` degrees of arc around (ra, dec) degrees."""

    shape = "CircularRegion"

    def __init__(self, ra, dec, radius):
        self.ra, self.dec, self.radius = float(ra), float(dec), float(radius)

    def contains(self, xcorners, ycorners, wcs, origin=0):
        """Index arrays of the pixels with a corner inside the circle.  The
        centre and radius are carried to pixel coordinates through the WCS
        (the radius along declination; square pixels assumed, as the
        reference does)."""
        xc, yc = wcs.all_world2pix(self.ra, self.dec, origin)
        xr, yr = wcs.all_world2pix(self.ra, self.dec + self.radius, origin)
        r2 = (xc - xr) ** 2 + (yc - yr) ** 2
        d2 = (xc - xcorners) ** 2 + (yc - ycorners) ** 2
        return np.where(np.any(d2 < r2, axis=-1))

    @property
    def bounding_box(self):
        """The (ra, dec) of the 4 corners of the RA/Dec-aligned square around
        the circle, shape (2, 4)."""
        dra = self.radius / np.cos(np.deg2rad(self.dec))
        ddec = self.radius
        corners = [(self.ra - dra, self.dec - ddec), (self.ra + dra, self.dec - ddec),
                   (self.ra + dra, self.dec + ddec), (self.ra - dra, self.dec + ddec)]
        return np.array(corners).T


class RectangularRegion:
    """The RA/Dec-aligned box [ra_min, ra_max] x [dec_min, dec_max] (degrees)."""

    shape = "RectangularRegion"

    def __init__(self, ra_min, ra_max, dec_min, dec_max):
        self.ra_min, self.ra_max = float(ra_min), float(ra_max)
        self.dec_min, self.dec_max = float(dec_min), float(dec_max)

    def contains(self, xcorners, ycorners, wcs, origin=0):
        ra, dec = wcs.all_pix2world(np.asarray(xcorners).ravel(), np.asarray(ycorners).ravel(), origin)
        ra = ra.reshape(np.shape(xcorners))
        dec = dec.reshape(np.shape(ycorners))
        inside = (ra > self.ra_min) & (ra < self.ra_max) & (dec > self.dec_min) & (dec < self.dec_max)
        return np.where(np.any(inside, axis=-1))

    @property
    def bounding_box(self):
        return np.array([(self.ra_min, self.dec_min), (self.ra_max, self.dec_min),
                         (self.ra_max, self.dec_max), (self.ra_min, self.dec_max)]).T
