"""Gnomonic (TAN) world coordinate systems and the local astrometry of a source.

forcepho takes each exposure's astrometry from an ``astropy.wcs.WCS`` and
linearises it at every source (``scale_at_sky``,
forcepho/utils/wcs.py:83-144; used by ``Patch._pack_astrometry``,
forcepho/patches/patch.py:301-337).  astropy is not a dependency here;
:class:`TanWCS` implements the FITS celestial WCS of the headers those
exposures carry -- ``RA---TAN``/``DEC--TAN`` with a ``CD`` or ``PC``+``CDELT``
matrix, no distortion -- from the published projection equations (Calabretta &
Greisen 2002, A&A 395, 1077: the zenithal TAN projection, eqs. 54-55, and the
spherical rotation of eqs. 2 and 5 with the native pole at theta_0 = 90 deg).
Pixel coordinates are 0-based, as astropy's ``*_values`` methods return them.
Headers with SIP or other distortion keywords are refused.

Both methods are vectorised over numpy arrays and computed in float64.
"""

import numpy as np

__all__ = ["TanWCS", "TanWCSStack", "scale_at_sky", "sky_to_pix"]

_D2R = np.pi / 180.0
_R2D = 180.0 / np.pi


class TanWCS:
    """A TAN projection from a FITS header (dict-like).

    Attributes: ``crpix`` (1-based, as in the header), ``crval`` (deg),
    ``cd`` (2x2, deg/pixel), ``lonpole`` (deg).
    """

    has_distortion = False

    def __init__(self, hdr):
        ct1, ct2 = str(hdr.get("CTYPE1", "")).strip(), str(hdr.get("CTYPE2", "")).strip()
        if not (ct1.startswith("RA---TAN") and ct2.startswith("DEC--TAN")):
            raise NotImplementedError(f"only RA---TAN/DEC--TAN is supported (got {ct1}, {ct2})")
        if ct1 != "RA---TAN" or ct2 != "DEC--TAN" or "A_ORDER" in hdr or "B_ORDER" in hdr:
            raise NotImplementedError("distortion (SIP, TPV, ...) is not supported")
        self.crpix = np.array([float(hdr["CRPIX1"]), float(hdr["CRPIX2"])])
        self.crval = np.array([float(hdr["CRVAL1"]), float(hdr["CRVAL2"])])
        if "CD1_1" in hdr:
            self.cd = np.array([[float(hdr.get("CD1_1", 0.0)), float(hdr.get("CD1_2", 0.0))],
                                [float(hdr.get("CD2_1", 0.0)), float(hdr.get("CD2_2", 0.0))]])
        else:
            pc = np.array([[float(hdr.get("PC1_1", 1.0)), float(hdr.get("PC1_2", 0.0))],
                           [float(hdr.get("PC2_1", 0.0)), float(hdr.get("PC2_2", 1.0))]])
            cdelt = np.array([float(hdr.get("CDELT1", 1.0)), float(hdr.get("CDELT2", 1.0))])
            self.cd = cdelt[:, None] * pc
        # default LONPOLE for a zenithal projection with delta_0 < theta_0 = 90
        self.lonpole = float(hdr.get("LONPOLE", 180.0 if self.crval[1] < 90.0 else 0.0))
        self.cdinv = np.linalg.inv(self.cd)
        self.naxis = (int(hdr.get("NAXIS1", 0)), int(hdr.get("NAXIS2", 0)))

    @property
    def pixel_scale_matrix(self):
        """deg per pixel (the CD matrix), as astropy's ``pixel_scale_matrix``."""
        return self.cd.copy()

    def pixel_to_world_values(self, x, y):
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        u = x + 1.0 - self.crpix[0]
        v = y + 1.0 - self.crpix[1]
        xi = self.cd[0, 0] * u + self.cd[0, 1] * v
        eta = self.cd[1, 0] * u + self.cd[1, 1] * v
        r = np.hypot(xi, eta)
        phi = np.arctan2(xi, -eta)
        theta = np.arctan2(_R2D, r)
        a0, d0 = self.crval * _D2R
        dphi = phi - self.lonpole * _D2R
        st, ct = np.sin(theta), np.cos(theta)
        sd0, cd0 = np.sin(d0), np.cos(d0)
        X = st * cd0 - ct * sd0 * np.cos(dphi)
        Y = -ct * np.sin(dphi)
        Z = st * sd0 + ct * cd0 * np.cos(dphi)
        ra = a0 + np.arctan2(Y, X)
        dec = np.arctan2(Z, np.hypot(X, Y))    # better conditioned than arcsin(Z)
        return np.mod(ra * _R2D, 360.0), dec * _R2D

    def world_to_pixel_values(self, ra, dec):
        ra = np.asarray(ra, dtype=np.float64) * _D2R
        dec = np.asarray(dec, dtype=np.float64) * _D2R
        a0, d0 = self.crval * _D2R
        da = ra - a0
        sd, cd = np.sin(dec), np.cos(dec)
        sd0, cd0 = np.sin(d0), np.cos(d0)
        X = sd * cd0 - cd * sd0 * np.cos(da)
        Y = -cd * np.sin(da)
        Z = sd * sd0 + cd * cd0 * np.cos(da)
        phi = self.lonpole * _D2R + np.arctan2(Y, X)
        r = _R2D * np.hypot(X, Y) / Z           # R_theta = cot(theta), theta = atan2(Z, |X, Y|)
        xi = r * np.sin(phi)
        eta = -r * np.cos(phi)
        u = self.cdinv[0, 0] * xi + self.cdinv[0, 1] * eta
        v = self.cdinv[1, 0] * xi + self.cdinv[1, 1] * eta
        return u + self.crpix[0] - 1.0, v + self.crpix[1] - 1.0

    # astropy's older names
    def all_pix2world(self, x, y, origin=0):
        return self.pixel_to_world_values(np.asarray(x) - origin, np.asarray(y) - origin)

    def all_world2pix(self, ra, dec, origin=0):
        x, y = self.world_to_pixel_values(ra, dec)
        return x + origin, y + origin


def scale_at_sky(sky, wcs, dpix=1.0, make_approx=False):
    """(CW, D) at sky = (ra, dec) in degrees: CW maps (dra, ddec) in degrees
    to pixels; D is pixels per arcsec.  Same two branches as the reference
    (forcepho/utils/wcs.py:83-144): for a WCS without distortion
    D = inv(3600 pixel_scale_matrix) and CW = 3600 D diag(cos dec, 1);
    otherwise (or with ``make_approx``) finite differences of ``dpix``
    pixels."""
    ra, dec = sky
    if getattr(wcs, "has_distortion", True) or make_approx:
        pos0_sky = np.array([ra, dec], dtype=np.float64)
        pos0_pix = np.array(wcs.world_to_pixel_values(*pos0_sky))
        pos1_sky = np.array(wcs.pixel_to_world_values(*(pos0_pix + np.array([dpix, 0.0]))))
        pos2_sky = np.array(wcs.pixel_to_world_values(*(pos0_pix + np.array([0.0, dpix]))))
        P = np.eye(2) * dpix
        St = np.array([pos1_sky - pos0_sky, pos2_sky - pos0_sky])
        CW_mat = np.linalg.solve(St, P).T
        Winv = np.eye(2)
        Winv[0, 0] = np.cos(np.deg2rad(pos0_sky[-1])) ** (-1)
        D_mat = 1.0 / 3600.0 * np.matmul(CW_mat, Winv)
    else:
        W = np.eye(2)
        W[0, 0] = np.cos(np.deg2rad(dec))
        D_mat = np.linalg.inv(wcs.pixel_scale_matrix * 3600.0)
        CW_mat = np.matmul(D_mat * 3600.0, W)
    return CW_mat, D_mat


def sky_to_pix(ra, dec, exp=None, ref_coords=0.0):
    """Pixel positions from the linearised astrometry of an exposure record
    with ``crval``, ``crpix`` and ``CW`` (forcepho/utils/wcs.py:147-178)."""
    crval, crpix, CW = exp["crval"][:], exp["crpix"][:], exp["CW"][:]
    if len(CW) != len(ra):
        CW, crval, crpix = CW[0], crval[0], crpix[0]
    sky = np.array([ra, dec]).T - (crval + ref_coords)
    return np.matmul(CW, sky[:, :, None])[..., 0] + crpix


class TanWCSStack:
    """Many TAN WCSs evaluated together: ``world_to_pixel_values(ra, dec)``
    maps k sky positions through each of n WCSs at once, returning (n, k)
    arrays -- the same formulas as :class:`TanWCS`, broadcast over a stack of
    parameters (used to test a region against every exposure of a store in
    one numpy pass)."""

    def __init__(self, wcses):
        self.crpix = np.array([w.crpix for w in wcses], dtype=np.float64).reshape(-1, 2)
        self.crval = np.array([w.crval for w in wcses], dtype=np.float64).reshape(-1, 2)
        self.cdinv = np.array([w.cdinv for w in wcses], dtype=np.float64).reshape(-1, 2, 2)
        self.lonpole = np.array([w.lonpole for w in wcses], dtype=np.float64)

    def __len__(self):
        return len(self.lonpole)

    def world_to_pixel_values(self, ra, dec):
        ra = np.atleast_1d(np.asarray(ra, dtype=np.float64))[None, :] * _D2R
        dec = np.atleast_1d(np.asarray(dec, dtype=np.float64))[None, :] * _D2R
        a0, d0 = self.crval[:, :1] * _D2R, self.crval[:, 1:] * _D2R
        da = ra - a0
        sd, cd = np.sin(dec), np.cos(dec)
        sd0, cd0 = np.sin(d0), np.cos(d0)
        X = sd * cd0 - cd * sd0 * np.cos(da)
        Y = -cd * np.sin(da)
        Z = sd * sd0 + cd * cd0 * np.cos(da)
        phi = self.lonpole[:, None] * _D2R + np.arctan2(Y, X)
        r = _R2D * np.hypot(X, Y) / Z
        xi = r * np.sin(phi)
        eta = -r * np.cos(phi)
        ci = self.cdinv
        u = ci[:, 0, 0, None] * xi + ci[:, 0, 1, None] * eta
        v = ci[:, 1, 0, None] * xi + ci[:, 1, 1, None] * eta
        return u + self.crpix[:, :1] - 1.0, v + self.crpix[:, 1:] - 1.0
