"""Gnomonic (TAN) world coordinate systems and the local astrometry of a source.

forcepho takes each exposure's astrometry from an ``astropy.wcs.WCS`` and
linearises it at every source (``scale_at_sky``,
forcepho/utils/wcs.py:83-144; used by ``Patch._pack_astrometry``,
forcepho/patches/patch.py:301-337).  astropy is not a dependency here;
:class:`TanWCS` implements the FITS celestial WCS of the headers those
exposures carry -- ``RA---TAN``/``DEC--TAN`` with a ``CD`` or ``PC``+``CDELT``
matrix, no distortion -- from the published projection equations (Calabretta &
Greisen 2002, A&A 395, 1077: the zenithal TAN projection, eqs. 54-55, and the
spherical rotation of eqs. 2 and 5 with the native pole at theta_0 = 90 deg),
with the SIP polynomial distortion convention (Shupe et al. 2005, ASP Conf.
Ser. 347, 491) for ``RA---TAN-SIP`` headers: (u, v) = pixel - CRPIX,
(xi, eta) = CD (u + f(u, v), v + g(u, v)) with f = sum A_p_q u^p v^q and
g = sum B_p_q u^p v^q.  The sky-to-pixel direction solves those polynomials
by Newton iteration to 1e-10 pixel, starting from the inverse polynomials
AP_p_q / BP_p_q when the header has them.  Pixel coordinates are 0-based, as
astropy's ``*_values`` methods return them.  Other distortions (TPV, lookup
tables) are refused.

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
        sip = ct1 == "RA---TAN-SIP" and ct2 == "DEC--TAN-SIP"
        if not sip and (ct1 != "RA---TAN" or ct2 != "DEC--TAN"):
            raise NotImplementedError(f"distortion {ct1}/{ct2} is not supported (TAN and TAN-SIP "
                                      "are)")
        if not sip and ("A_ORDER" in hdr or "B_ORDER" in hdr):
            raise NotImplementedError("SIP coefficients without a -SIP projection code")
        self.sip = _read_sip(hdr) if sip else None
        self.has_distortion = self.sip is not None
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
        if self.sip is not None:
            u, v = u + _poly(self.sip["A"], u, v), v + _poly(self.sip["B"], u, v)
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
        if self.sip is not None:
            u, v = _sip_invert(self.sip, u, v)
        return u + self.crpix[0] - 1.0, v + self.crpix[1] - 1.0

    # astropy's older names
    def all_pix2world(self, x, y, origin=0):
        return self.pixel_to_world_values(np.asarray(x) - origin, np.asarray(y) - origin)

    def all_world2pix(self, ra, dec, origin=0):
        x, y = self.world_to_pixel_values(ra, dec)
        return x + origin, y + origin


def _read_sip(hdr):
    """SIP coefficient tables {name: {(p, q): value}} for A, B (and AP, BP if
    present) from a header."""
    out = {}
    for name in ("A", "B", "AP", "BP"):
        order = hdr.get(f"{name}_ORDER")
        if order is None:
            if name in ("A", "B"):
                raise ValueError(f"TAN-SIP header without {name}_ORDER")
            continue
        coef = {}
        for p in range(int(order) + 1):
            for q in range(int(order) + 1 - p):
                c = hdr.get(f"{name}_{p}_{q}")
                if c:
                    coef[(p, q)] = float(c)
        out[name] = coef
    return out


def _poly(coef, u, v):
    """sum over (p, q) of coef * u^p v^q."""
    out = np.zeros(np.broadcast(u, v).shape)
    for (p, q), c in coef.items():
        out = out + c * u ** p * v ** q
    return out


def _poly_grad(coef, u, v):
    du = np.zeros(np.broadcast(u, v).shape)
    dv = np.zeros_like(du)
    for (p, q), c in coef.items():
        if p:
            du = du + c * p * u ** (p - 1) * v ** q
        if q:
            dv = dv + c * q * u ** p * v ** (q - 1)
    return du, dv


def _sip_invert(sip, U, V, tol=1e-10, max_iter=50):
    """(u, v) with u + f(u, v) = U, v + g(u, v) = V (Newton iteration from the
    inverse polynomials, or from (U, V))."""
    U = np.asarray(U, dtype=np.float64)
    V = np.asarray(V, dtype=np.float64)
    if "AP" in sip and "BP" in sip:
        u, v = U + _poly(sip["AP"], U, V), V + _poly(sip["BP"], U, V)
    else:
        u, v = U.copy(), V.copy()
    for _ in range(max_iter):
        fu, gu = u + _poly(sip["A"], u, v) - U, v + _poly(sip["B"], u, v) - V
        if np.all(np.abs(fu) < tol) and np.all(np.abs(gu) < tol):
            break
        adu, adv = _poly_grad(sip["A"], u, v)
        bdu, bdv = _poly_grad(sip["B"], u, v)
        j11, j12, j21, j22 = 1.0 + adu, adv, bdu, 1.0 + bdv
        det = j11 * j22 - j12 * j21
        u = u - (j22 * fu - j12 * gu) / det
        v = v - (j11 * gu - j21 * fu) / det
    return u, v


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
        self.wcses = list(wcses)
        self.distorted = any(getattr(w, "has_distortion", False) for w in self.wcses)
        self.crpix = np.array([w.crpix for w in wcses], dtype=np.float64).reshape(-1, 2)
        self.crval = np.array([w.crval for w in wcses], dtype=np.float64).reshape(-1, 2)
        self.cdinv = np.array([w.cdinv for w in wcses], dtype=np.float64).reshape(-1, 2, 2)
        self.lonpole = np.array([w.lonpole for w in wcses], dtype=np.float64)

    def __len__(self):
        return len(self.lonpole)

    def world_to_pixel_values(self, ra, dec):
        if self.distorted:      # SIP: one WCS at a time
            xy = [w.world_to_pixel_values(np.atleast_1d(ra), np.atleast_1d(dec))
                  for w in self.wcses]
            return (np.array([p[0] for p in xy]).reshape(len(xy), -1),
                    np.array([p[1] for p in xy]).reshape(len(xy), -1))
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
