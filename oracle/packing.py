"""CPU restatement of forcepho's super-pixel selection and pixel packing.
TEST INFRASTRUCTURE ONLY: tests/ and bench.py's CPU-baseline leg use it as
the checker of the device store (forcepho_b200/csrc/fpho_store.cu); the
forcepho_b200 product never imports it.

Given each exposure's super-pixel array (nsx, nsy, 2 s^2) and the region test
in that exposure's pixels, ``pack`` returns what forcepho's
``StorePatch.find_pixels`` + ``PixelPatch.pack_pix`` + ``_cap_snr`` produce:

  * super-pixel corners (0,0), (1,0), (1,1), (0,1) times (s-1) from the
    first pixel (forcepho/patches/storage.py:117-139);
  * circle: any corner with (xc-x)^2 + (yc-y)^2 < r2 in float64
    (forcepho/region.py:91-116); rectangle: any corner whose TAN sky
    position is strictly inside the box (region.py:168-192);
  * selected super-pixels in numpy.where (row-major) order; fluxes
    data[sx, sy, :s^2], inverse errors data[sx, sy, s^2:], coordinates
    x = sx s + k // s, y = sy s + k % s (storage.py:141-149, 245-276;
    pixel_patch.py:307-342);
  * exposures concatenated in the given order, the background offset
    subtracted in float32 (pixel_patch.py:171-178), then ierr capped at
    max_snr / data where data * ierr > max_snr (pixel_patch.py:200-205).

The rectangle test uses the same TAN projection formulas as the product
(Calabretta & Greisen 2002, eqs. 2, 5, 54-55) in float64 numpy.

Pinned against the reference's own packing code by
tests/golden/packing_store.npz (tests/test_packing.py).
"""

import numpy as np

_D2R = np.pi / 180.0
_R2D = 180.0 / np.pi


def superpixel_corners(nsx, nsy, s):
    """(nsx, nsy, 4) x and y of the four corner pixels."""
    sx, sy = np.meshgrid(np.arange(nsx), np.arange(nsy), indexing="ij")
    off = np.array([(0, 0), (1, 0), (1, 1), (0, 1)]) * (s - 1)
    x = sx[..., None] * s + off[:, 0]
    y = sy[..., None] * s + off[:, 1]
    return x.astype(np.int64), y.astype(np.int64)


def _tan_pix2world(x, y, p):
    crpix1, crpix2, cd11, cd12, cd21, cd22, crval1, crval2, lonpole = p[4:13]
    u = x + 1.0 - crpix1
    v = y + 1.0 - crpix2
    xi = cd11 * u + cd12 * v
    eta = cd21 * u + cd22 * v
    r = np.hypot(xi, eta)
    phi = np.arctan2(xi, -eta)
    theta = np.arctan2(_R2D, r)
    dphi = phi - lonpole * _D2R
    a0, d0 = crval1 * _D2R, crval2 * _D2R
    st, ct = np.sin(theta), np.cos(theta)
    sd0, cd0 = np.sin(d0), np.cos(d0)
    X = st * cd0 - ct * sd0 * np.cos(dphi)
    Y = -ct * np.sin(dphi)
    Z = st * sd0 + ct * cd0 * np.cos(dphi)
    ra = np.mod((a0 + np.arctan2(Y, X)) * _R2D, 360.0)
    dec = np.arctan2(Z, np.hypot(X, Y)) * _R2D
    return ra, dec


def select(kind, p, nsx, nsy, s):
    """(sx, sy) of the selected super-pixels (np.where order)."""
    x, y = superpixel_corners(nsx, nsy, s)
    if kind == 1:
        xc, yc, r2 = p[0], p[1], p[2]
        d2 = (xc - x) ** 2 + (yc - y) ** 2
        return np.where(np.any(d2 < r2, axis=-1))
    ra, dec = _tan_pix2world(x.astype(np.float64), y.astype(np.float64), p)
    ok = (ra > p[0]) & (ra < p[1]) & (dec > p[2]) & (dec < p[3])
    return np.where(np.any(ok, axis=-1))


def pack(superpixels, regions, background=None, max_snr=None):
    """superpixels: list of (nsx, nsy, 2 s^2) float32 arrays (one per listed
    exposure); regions: list of (kind, params).  Returns dict(data, ierr, xpix,
    ypix, exposure_start, exposure_N)."""
    data, ierr, xpix, ypix, N = [], [], [], [], []
    for e, (sp, (kind, p)) in enumerate(zip(superpixels, regions)):
        nsx, nsy, two_s2 = sp.shape
        s2 = two_s2 // 2
        s = int(round(np.sqrt(s2)))
        sx, sy = select(kind, np.asarray(p, dtype=np.float64), nsx, nsy, s)
        k = np.arange(s2)
        d = sp[sx, sy, :s2].reshape(-1)
        if background is not None:
            d = d - np.float32(background[e])
        data.append(d)
        ierr.append(sp[sx, sy, s2:].reshape(-1))
        xpix.append((sx[:, None] * s + k[None, :] // s).reshape(-1))
        ypix.append((sy[:, None] * s + k[None, :] % s).reshape(-1))
        N.append(len(sx) * s2)
    out = dict(data=np.concatenate(data).astype(np.float32),
               ierr=np.concatenate(ierr).astype(np.float32),
               xpix=np.concatenate(xpix).astype(np.float32),
               ypix=np.concatenate(ypix).astype(np.float32),
               exposure_N=np.array(N, dtype=np.int32))
    out["exposure_start"] = np.concatenate([[0], np.cumsum(N)[:-1]]).astype(np.int32)
    if max_snr:
        m = np.float32(max_snr)
        cap = (out["ierr"] > 0) & (out["data"] * out["ierr"] > m)
        out["ierr"][cap] = m / out["data"][cap]
    return out
