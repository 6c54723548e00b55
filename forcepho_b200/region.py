"""Sky regions that select the pixels of a patch.

Same classes and selection rules as forcepho/region.py:16-300: a
:class:`CircularRegion` keeps every super-pixel with at least one corner
pixel strictly closer to the centre (in pixels of the exposure, radius taken
along declination) than the radius; a :class:`RectangularRegion` keeps every
super-pixel with a corner strictly inside the RA/Dec box.  ``contains``
returns ``np.where`` of the selection, so super-pixels come in row-major
(x super-pixel, y super-pixel) order.

The device store (:mod:`forcepho_b200.patches.device_store`) evaluates the
same tests in a CUDA kernel from :meth:`Region.device_params`.
"""

import numpy as np

__all__ = ["Region", "CircularRegion", "RectangularRegion", "polygons_overlap",
           "polygon_contains"]

REGION_CIRCLE, REGION_RECT = 1, 2


class Region:
    """Base class: selects nothing."""

    shape = "Region"

    def contains(self, x, y, wcs):
        return np.zeros(len(x), dtype=bool)

    @property
    def bounding_box(self):
        return None

    def overlaps(self, hdr, wcs=None):
        """Whether the RA/Dec bounding box of an image (its header's NAXIS
        and WCS) overlaps this region's bounding box
        (forcepho/region.py:48-62)."""
        from .wcs import TanWCS
        wcs = wcs or TanWCS(hdr)
        nx, ny = hdr["NAXIS1"], hdr["NAXIS2"]
        ira, idec = wcs.pixel_to_world_values(np.array([0, nx, nx, 0]), np.array([0, 0, ny, ny]))
        return polygons_overlap(self, RectangularRegion(ira.min(), ira.max(), idec.min(),
                                                        idec.max()))


class CircularRegion(Region):
    """A circle of ``radius`` degrees of arc around (ra, dec) in degrees."""

    def __init__(self, ra, dec, radius):
        self.ra, self.dec, self.radius = ra, dec, radius
        self.shape = "CircularRegion"

    def pixel_circle(self, wcs):
        """(xc, yc, r2): centre and squared radius in pixels of `wcs`, as
        forcepho/region.py:110-113 derives them."""
        xc, yc = wcs.world_to_pixel_values(self.ra, self.dec)
        xr, yr = wcs.world_to_pixel_values(self.ra, self.dec + self.radius)
        return float(xc), float(yc), float((xc - xr) ** 2 + (yc - yr) ** 2)

    def contains(self, xcorners, ycorners, wcs):
        xc, yc, r2 = self.pixel_circle(wcs)
        d2 = (xc - xcorners) ** 2 + (yc - ycorners) ** 2
        return np.where(np.any(d2 < r2, axis=-1))

    def device_params(self, wcs):
        xc, yc, r2 = self.pixel_circle(wcs)
        return REGION_CIRCLE, [xc, yc, r2]

    @property
    def bounding_box(self):
        dra = self.radius / np.cos(np.deg2rad(self.dec))
        ddec = self.radius
        corners = [(self.ra - dra, self.dec - ddec), (self.ra + dra, self.dec - ddec),
                   (self.ra + dra, self.dec + ddec), (self.ra - dra, self.dec + ddec)]
        return np.array(corners).T


class RectangularRegion(Region):
    """An RA/Dec-aligned box (degrees)."""

    def __init__(self, ra_min, ra_max, dec_min, dec_max):
        self.ra_min, self.ra_max = ra_min, ra_max
        self.dec_min, self.dec_max = dec_min, dec_max
        self.shape = "RectangularRegion"

    def contains(self, xcorners, ycorners, wcs):
        ra, dec = wcs.pixel_to_world_values(xcorners, ycorners)
        valid = ((ra > self.ra_min) & (ra < self.ra_max) &
                 (dec > self.dec_min) & (dec < self.dec_max))
        return np.where(np.any(valid, axis=-1))

    def device_params(self, wcs):
        """The box and the TAN parameters the kernel needs to map corners to
        the sky: crpix (1-based), CD, crval, lonpole.  The kernel maps pixels
        with the TAN projection alone, so distorted (SIP) WCSs are refused."""
        if getattr(wcs, "has_distortion", False):
            raise NotImplementedError("RA/Dec boxes on the device need an undistorted TAN WCS")
        p = [self.ra_min, self.ra_max, self.dec_min, self.dec_max,
             wcs.crpix[0], wcs.crpix[1], wcs.cd[0, 0], wcs.cd[0, 1], wcs.cd[1, 0], wcs.cd[1, 1],
             wcs.crval[0], wcs.crval[1], wcs.lonpole]
        return REGION_RECT, p

    @property
    def bounding_box(self):
        corners = [(self.ra_min, self.dec_min), (self.ra_max, self.dec_min),
                   (self.ra_max, self.dec_max), (self.ra_min, self.dec_max)]
        return np.array(corners).T


def polygons_overlap(a, b):
    """Whether the (convex, consistently ordered) bounding polygons of two
    regions intersect, touching included: no edge normal of either polygon
    separates their projections (the separating-axis test of
    forcepho/region.py:214-264)."""
    ax, ay = a.bounding_box
    bx, by = b.bounding_box
    for xs, ys in (a.bounding_box, b.bounding_box):
        n = len(xs)
        i = np.arange(n)
        nx, ny = ys[(i + 1) % n] - ys[i], xs[i] - xs[(i + 1) % n]
        pa = nx[:, None] * ax[None, :] + ny[:, None] * ay[None, :]
        pb = nx[:, None] * bx[None, :] + ny[:, None] * by[None, :]
        if np.any((pa.max(-1) < pb.min(-1)) | (pb.max(-1) < pa.min(-1))):
            return False
    return True


def polygon_contains(poly, points):
    """Whether each point (n, 2) is inside a convex polygon (m, 2) given in
    either winding: the cross products of every edge with the point have one
    sign (forcepho/region.py:267-302; a point on an edge gives a zero and
    is outside)."""
    poly = np.asarray(poly, dtype=np.float64)
    points = np.atleast_2d(np.asarray(points, dtype=np.float64))
    edges = np.diff(np.vstack([poly, poly[:1]]), axis=0)
    rel = points[:, None, :] - poly[None, :, :]
    sign = np.sign(edges[:, 0] * rel[:, :, 1] - edges[:, 1] * rel[:, :, 0])
    return np.all(sign == sign[:, :1], axis=1)
