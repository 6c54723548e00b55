"""Seeded synthetic patches in the reference's packed layout.

No public dataset is involved in forcepho's hot path; its inputs are packed
patches (pixel data, inverse errors and pixel coordinates per exposure,
per-exposure astrometry, photometric conversion and PSF mixtures) and source
proposals.  This module draws them from ``numpy.random.default_rng(seed)``
with the distributions of the workloads the benchmarks and tests use:

  "single"    1 band x 1 exposure of 64x64 px, 1 source, 3-Gaussian PSF
  "field20"   8 bands x 4 exposures of 128x128 px, 20 sources, 5-Gaussian
              PSFs, per-exposure rotation (+-1 deg), scale (+-2%), flux
              calibration U[0.8, 1.2], 2% of pixels masked (ierr = 0)
  "uneven"    n patches (256 by default): sources U{1..30}, bands U{1..8},
              exposures per band U{1..8}, exposure side U[32, 200] px
  "stress60"  60 sources (half with sersic in [3.5, 6], rh up to 1 arcsec,
              fluxes LogNormal(0, 3)), 15 bands x 6 exposures of 256x256 px,
              6-Gaussian PSFs

Pixel scale 0.03 arcsec/px.  D (pixels per arcsec) and CW (pixels per degree,
CW = D diag(3600 cos dec0, 3600)) follow forcepho/slow/stamp.py:250-254.
Pixels are packed per exposure in 8x8 superpixels ordered along a Morton
curve, each exposure padded to whole superpixels with pixels at x = y = -1 and
ierr = 0 (the reference's padding convention, forcepho/patches/pixel_patch.py
:472-483).  The PSF mixture of an exposure is repeated for every Sersic radius
bin (sersic_bin = 0..n_radii-1) and every source.  Data are the truth model
plus Gaussian noise of sigma = 0.05 x the exposure's peak, ierr = 1/sigma.
Proposals are evaluated at the truth perturbed by 1% in every parameter.
"""

from dataclasses import dataclass, field

import numpy as np

from .patches.patch import PSF_DTYPE, PatchBase
from .patches.device_patch import GPUPatchMixin
from .sources import default_table, proposal_from_params

__all__ = ["PatchSpec", "SyntheticPatch", "make_workload", "make_patch", "workload_spec",
           "render_model_numpy", "PIXEL_SCALE", "DEC0"]

PIXEL_SCALE = 0.03      # arcsec per pixel
DEC0 = -27.78           # declination of the patch centre (degrees)


@dataclass
class PatchSpec:
    n_sources: int
    exposures_per_band: list          # exposures of each band
    shapes: list                      # (nx, ny) per exposure
    n_psf: int = 3                    # PSF Gaussians per exposure
    psf_sigma: tuple = (0.5, 3.0)     # PSF component sigma range (px)
    rot_deg: float = 0.0              # per-exposure rotation amplitude
    scale_frac: float = 0.0           # per-exposure pixel-scale amplitude
    g_range: tuple = (1.0, 1.0)       # photometric conversion range
    mask_frac: float = 0.0            # fraction of pixels with ierr = 0
    flux_sigma: float = 1.0           # LogNormal sigma of fluxes
    position: str = "uniform"         # "centre" (+-0.3") or "uniform" over the patch
    sersic: tuple = (1.0, 5.0)
    rh: tuple = (0.05, 0.3)
    bright_fraction: float = 0.0      # fraction drawn from sersic/rh "bright" ranges
    bright_sersic: tuple = (3.5, 6.0)
    bright_rh: tuple = (0.05, 1.0)
    perturb: float = 0.01
    extra: dict = field(default_factory=dict)

    @property
    def n_bands(self):
        return len(self.exposures_per_band)


WORKLOADS = ("single", "field20", "uneven", "stress60")


def workload_spec(name, rng=None):
    """PatchSpec of a workload ("uneven" draws one spec per patch from
    ``rng``, see :func:`make_workload`)."""
    if name == "single":
        return PatchSpec(n_sources=1, exposures_per_band=[1], shapes=[(64, 64)], n_psf=3,
                         psf_sigma=(0.5, 3.0), flux_sigma=1.0, position="centre")
    if name == "field20":
        return PatchSpec(n_sources=20, exposures_per_band=[4] * 8, shapes=[(128, 128)] * 32,
                         n_psf=5, psf_sigma=(0.5, 4.0), rot_deg=1.0, scale_frac=0.02,
                         g_range=(0.8, 1.2), mask_frac=0.02, flux_sigma=1.5)
    if name == "uneven":
        rng = rng or np.random.default_rng(0)
        nb = int(rng.integers(1, 9))
        epb = [int(rng.integers(1, 9)) for _ in range(nb)]
        shapes = []
        for _ in range(sum(epb)):
            side = int(np.round(rng.uniform(32, 200)))
            shapes.append((side, side))
        return PatchSpec(n_sources=int(rng.integers(1, 31)), exposures_per_band=epb,
                         shapes=shapes, n_psf=5, psf_sigma=(0.5, 4.0), rot_deg=1.0,
                         scale_frac=0.02, g_range=(0.8, 1.2), mask_frac=0.02, flux_sigma=1.5)
    if name == "stress60":
        return PatchSpec(n_sources=60, exposures_per_band=[6] * 15, shapes=[(256, 256)] * 90,
                         n_psf=6, psf_sigma=(0.5, 4.0), rot_deg=1.0, scale_frac=0.02,
                         g_range=(0.8, 1.2), mask_frac=0.02, flux_sigma=3.0,
                         bright_fraction=0.5, bright_sersic=(3.5, 6.0), bright_rh=(0.05, 1.0))
    raise ValueError(f"unknown workload {name!r} (one of {WORKLOADS})")


class SyntheticPatch(PatchBase, GPUPatchMixin):
    """A packed synthetic patch with its truth and perturbed parameters.

    Attributes beyond the PatchBase arrays: ``spec``, ``table`` (SersicTable),
    ``truth`` and ``params`` (n_sources x (n_bands + 6) in Scene order),
    ``original_shapes`` and ``original_sizes`` per exposure."""

    def __init__(self, return_residual=False):
        PatchBase.__init__(self, return_residual=return_residual)
        self.device_patch = None

    @property
    def n_sources_(self):
        return self.n_sources

    def proposal(self, params=None):
        p = self.params if params is None else params
        return proposal_from_params(p, self.n_bands, self.table)

    def truth_proposal(self):
        return proposal_from_params(self.truth, self.n_bands, self.table)

    # ---- scenes: subsets of the patch's sources with their own metadata
    def set_scene(self, indices, params=None):
        """A scene of the sources `indices` (rows of ``truth``), with
        parameters `params` (len(indices) x (n_bands + 6); default the
        perturbed ``params`` rows), as the reference's ``set_scene``
        (forcepho/patches/pixel_patch.py) builds one from catalog rows."""
        from .sources import Scene
        idx = np.atleast_1d(np.asarray(indices, dtype=np.int64))
        p = self.params[idx] if params is None else np.asarray(params, np.float64)
        sc = Scene(len(idx), self.n_bands, self.table, params=p)
        sc.source_indices = idx
        return sc

    def pack_meta(self, scene):
        """Pack the per-source metadata (astrometry and PSF rows) of `scene`
        into the patch arrays, as the reference's ``pack_meta``
        (forcepho/patches/patch.py:242-396); pixel arrays are untouched."""
        full = self._meta_full
        idx = scene.source_indices
        ns, n_exp = len(idx), len(self.exposure_N)
        self.n_sources = ns
        self.D = np.ascontiguousarray(full["D"][:, idx])
        self.CW = np.ascontiguousarray(full["CW"][:, idx])
        self.crpix = np.ascontiguousarray(full["crpix"][:, idx])
        self.crval = np.ascontiguousarray(full["crval"][:, idx])
        npsf = full["npsf"]
        self.psfgauss = np.concatenate([np.tile(m, ns) for m in full["mix"]]).astype(PSF_DTYPE)
        self.psfgauss_start = (np.arange(n_exp) * ns * npsf).astype(np.int32)
        self.coerce_arrays()

    @property
    def pairs_per_eval(self):
        """Nominal (pixel, image Gaussian) pairs of one evaluation: every
        pixel (padding included) times the Gaussians of its exposure."""
        npsf_e = np.repeat(self.n_psf_per_source, self.band_N.astype(np.int64))
        return int(np.sum(self.exposure_N.astype(np.int64) * npsf_e * self.n_sources))


def _morton_order(nsx, nsy):
    sx, sy = np.meshgrid(np.arange(nsx), np.arange(nsy), indexing="ij")
    sx, sy = sx.ravel(), sy.ravel()

    def spread(v):
        v = v.astype(np.uint64)
        out = np.zeros_like(v)
        for b in range(16):
            out |= ((v >> np.uint64(b)) & np.uint64(1)) << np.uint64(2 * b)
        return out

    code = spread(sx) | (spread(sy) << np.uint64(1))
    o = np.argsort(code, kind="stable")
    return sx[o], sy[o]


def _pack_exposure_pixels(nx, ny):
    """x, y, valid arrays of one exposure in Morton-ordered 8x8 superpixels."""
    nsx, nsy = (nx + 7) // 8, (ny + 7) // 8
    sx, sy = _morton_order(nsx, nsy)
    iy, ix = np.meshgrid(np.arange(8), np.arange(8), indexing="ij")
    x = (sx[:, None] * 8 + ix.ravel()[None, :]).ravel()
    y = (sy[:, None] * 8 + iy.ravel()[None, :]).ravel()
    valid = (x < nx) & (y < ny)
    return x, y, valid


def _rot(t):
    c, s = np.cos(t), np.sin(t)
    return np.array([[c, -s], [s, c]])


def render_model_numpy(patch, params, nsigma=7.0):
    """FP64 model image (flat, patch pixel order) of Scene-ordered params,
    with the second-order pixel-integration correction and no cutoff other
    than truncating each Gaussian at ``nsigma`` (used only to synthesise data)."""
    table = patch.table
    nb = patch.n_bands
    params = np.asarray(params, dtype=np.float64).reshape(-1, nb + 6)
    model = np.zeros(patch.npix, dtype=np.float64)
    rad2 = table.radii ** 2
    for b in range(nb):
        for e in range(int(patch.band_start[b]), int(patch.band_start[b] + patch.band_N[b])):
            p0, n = int(patch.exposure_start[e]), int(patch.exposure_N[e])
            xs = patch.xpix[p0:p0 + n].astype(np.float64)
            ys = patch.ypix[p0:p0 + n].astype(np.float64)
            npsf = int(patch.n_psf_per_source[b])
            psf = patch.psfgauss[int(patch.psfgauss_start[e]):int(patch.psfgauss_start[e]) + npsf]
            for s, p in enumerate(params):
                flux, (ra, dec, q, pa, nser, rh) = p[b], p[nb:]
                amps = table.amplitudes(nser, rh)
                D = patch.D[e, s].astype(np.float64)
                CW = patch.CW[e, s].astype(np.float64)
                T = D @ _rot(pa) @ np.diag([1.0 / q, q])
                cen = CW @ (np.array([ra, dec]) - patch.crval[e, s]) + patch.crpix[e, s]
                for row in psf:
                    k = int(row["sersic_bin"])
                    Sig = rad2[k] * T @ T.T + np.array([[row["Cxx"], row["Cxy"]],
                                                        [row["Cxy"], row["Cyy"]]])
                    F = np.linalg.inv(Sig)
                    A = patch.G[e] * row["amp"] * np.sqrt(np.linalg.det(F)) / (2 * np.pi) \
                        * flux * amps[k]
                    xc, yc = cen[0] + row["xcen"], cen[1] + row["ycen"]
                    wx, wy = nsigma * np.sqrt(Sig[0, 0]), nsigma * np.sqrt(Sig[1, 1])
                    m = (np.abs(xs - xc) < wx) & (np.abs(ys - yc) < wy)
                    if not m.any():
                        continue
                    dx, dy = xs[m] - xc, ys[m] - yc
                    vx = F[0, 0] * dx + F[0, 1] * dy
                    vy = F[1, 1] * dy + F[0, 1] * dx
                    H = 1 + (vx * vx + vy * vy - F[0, 0] - F[1, 1]) / 24.0
                    model[p0:p0 + n][m] += A * np.exp(-0.5 * (dx * vx + dy * vy)) * H
    return model


def render_model_gpu(patch, params):
    """Model image of Scene-ordered params evaluated by the CUDA path itself
    (residual output with zero data: model = -residual)."""
    from .proposal import GPUProposer
    data, ierr = patch.data, patch.ierr
    patch.data = np.zeros_like(patch.xpix)
    patch.ierr = np.ones_like(patch.xpix)
    orig = patch.return_residual
    patch.return_residual = True
    try:
        patch.send_to_device()
        prop = proposal_from_params(params, patch.n_bands, patch.table)
        _, _, res = GPUProposer().evaluate_proposal(prop, patch=patch, unpack=False)
    finally:
        patch.free()
        patch.data, patch.ierr = data, ierr
        patch.return_residual = orig
    return -res.astype(np.float64)


def make_patch(spec, seed=0, table=None, render=None, return_residual=False):
    """Draw a SyntheticPatch from ``spec``.

    ``render(patch, params) -> flat model`` synthesises the truth image
    (default :func:`render_model_numpy`); the data are that model plus noise.
    """
    rng = np.random.default_rng(seed)
    table = table or default_table()
    nb, ns = spec.n_bands, spec.n_sources
    n_exp = sum(spec.exposures_per_band)
    assert len(spec.shapes) == n_exp
    P = SyntheticPatch(return_residual=return_residual)
    P.spec, P.table = spec, table

    # --- per-exposure astrometry (linear WCS about the patch centre)
    cosd = np.cos(np.deg2rad(DEC0))
    Dexp, CWexp, crpix0 = [], [], []
    for e in range(n_exp):
        phi = np.deg2rad(rng.uniform(-spec.rot_deg, spec.rot_deg)) if spec.rot_deg else 0.0
        scl = 1.0 + (rng.uniform(-spec.scale_frac, spec.scale_frac) if spec.scale_frac else 0.0)
        D = _rot(phi) / (PIXEL_SCALE * scl)
        Dexp.append(D)
        CWexp.append(D @ np.diag([3600.0 * cosd, 3600.0]))
        nx, ny = spec.shapes[e]
        crpix0.append(np.array([(nx - 1) / 2.0, (ny - 1) / 2.0]))
    G = rng.uniform(*spec.g_range, size=n_exp) if spec.g_range[0] != spec.g_range[1] \
        else np.full(n_exp, spec.g_range[0])

    # --- sources (Scene order: fluxes, ra, dec, q, pa, sersic, rhalf)
    nx0, ny0 = spec.shapes[0]
    truth = np.zeros((ns, nb + 6))
    for s in range(ns):
        bright = rng.uniform() < spec.bright_fraction
        nser = rng.uniform(*(spec.bright_sersic if bright else spec.sersic))
        rh = rng.uniform(*(spec.bright_rh if bright else spec.rh))
        q = rng.uniform(0.4, 1.0)
        pa = rng.uniform(-np.pi / 2, np.pi / 2)
        if spec.position == "centre":
            off = rng.uniform(-0.3, 0.3, size=2)  # arcsec
        else:
            half = 0.45 * np.array([nx0, ny0]) * PIXEL_SCALE
            off = rng.uniform(-half, half)
        ra = off[0] / 3600.0 / cosd
        dec = off[1] / 3600.0
        fluxes = rng.lognormal(0.0, spec.flux_sigma, size=nb)
        truth[s] = np.concatenate([fluxes, [ra, dec, q, pa, nser, rh]])
    P.truth = truth
    P.params = truth * (1.0 + spec.perturb)

    # --- pixels
    xs, ys, valid, exp_start, exp_n = [], [], [], [], []
    i = 0
    for e in range(n_exp):
        x, y, v = _pack_exposure_pixels(*spec.shapes[e])
        x = np.where(v, x, -1).astype(np.float32)
        y = np.where(v, y, -1).astype(np.float32)
        xs.append(x); ys.append(y); valid.append(v)
        exp_start.append(i); exp_n.append(len(x))
        i += len(x)
    npix = i
    P.build_patch(npix=npix, n_sources=ns, n_radii=table.n_radii, n_bands=nb, n_exp=n_exp)
    P.xpix[:] = np.concatenate(xs)
    P.ypix[:] = np.concatenate(ys)
    P.exposure_start[:] = exp_start
    P.exposure_N[:] = exp_n
    P.band_N[:] = spec.exposures_per_band
    P.band_start[:] = np.concatenate([[0], np.cumsum(spec.exposures_per_band)[:-1]])
    P.original_shapes = [tuple(s) for s in spec.shapes]
    P.original_sizes = [int(a * b) for a, b in spec.shapes]
    validall = np.concatenate(valid)

    # --- metadata: per (exposure, source) astrometry packed at the truth position
    P.rad2[:] = table.rad2
    for e in range(n_exp):
        for s in range(ns):
            sky = truth[s, nb:nb + 2]
            P.D[e, s] = Dexp[e]
            P.CW[e, s] = CWexp[e]
            P.crval[e, s] = sky
            P.crpix[e, s] = crpix0[e] + CWexp[e] @ sky
    P.G[:] = G

    # --- PSF: one mixture per exposure, repeated per radius bin and source
    nr = table.n_radii
    npsf = nr * spec.n_psf
    P.n_psf_per_source[:] = npsf
    rows, mixes = [], []
    P.psfgauss_start[:] = np.arange(n_exp) * ns * npsf
    for e in range(n_exp):
        sig = rng.uniform(*spec.psf_sigma, size=spec.n_psf)
        amp = rng.dirichlet(np.ones(spec.n_psf))
        ell = rng.uniform(-0.1, 0.1, size=spec.n_psf)
        cxy = rng.uniform(-0.05, 0.05, size=spec.n_psf) * sig ** 2
        off = rng.normal(0.0, 0.05, size=(spec.n_psf, 2))
        mix = np.zeros(spec.n_psf, dtype=PSF_DTYPE)
        mix["amp"], mix["xcen"], mix["ycen"] = amp, off[:, 0], off[:, 1]
        mix["Cxx"], mix["Cyy"], mix["Cxy"] = sig ** 2 * (1 + ell), sig ** 2 * (1 - ell), cxy
        per_source = np.concatenate([mix.copy() for _ in range(nr)])
        per_source["sersic_bin"] = np.repeat(np.arange(nr), spec.n_psf)
        rows.append(np.tile(per_source, ns))
        mixes.append(per_source)
    P.psfgauss = np.concatenate(rows).astype(PSF_DTYPE)
    P._meta_full = {"D": P.D.copy(), "CW": P.CW.copy(), "crpix": P.crpix.copy(),
                    "crval": P.crval.copy(), "mix": mixes, "npsf": npsf}

    # --- data: truth + noise; ierr = 1/sigma per exposure; masked pixels
    model = (render or render_model_numpy)(P, truth)
    data = np.zeros(npix, dtype=np.float64)
    ierr = np.zeros(npix, dtype=np.float64)
    for e in range(n_exp):
        sl = slice(exp_start[e], exp_start[e] + exp_n[e])
        m = model[sl]
        v = validall[sl]
        peak = max(np.max(m[v]) if v.any() else 0.0, 1e-12)
        sigma = 0.05 * peak
        d = m + rng.normal(0.0, sigma, size=m.shape)
        ie = np.full(m.shape, 1.0 / sigma)
        if spec.mask_frac:
            ie[rng.uniform(size=m.shape) < spec.mask_frac] = 0.0
        d[~v] = 0.0
        ie[~v] = 0.0
        data[sl], ierr[sl] = d, ie
    P.data[:] = data.astype(np.float32)
    P.ierr[:] = ierr.astype(np.float32)
    P.coerce_arrays()
    P._dirty_data = True
    return P


def make_workload(name, seed=0, render=None, return_residual=False, n_patches=256):
    """The patch of a workload (for "uneven", a list of ``n_patches``)."""
    if name == "uneven":
        rng = np.random.default_rng(seed)
        out = []
        for i in range(n_patches):
            spec = workload_spec("uneven", rng)
            out.append(make_patch(spec, seed=int(rng.integers(2 ** 31)), render=render,
                                  return_residual=return_residual))
        return out
    return make_patch(workload_spec(name), seed=seed, render=render,
                      return_residual=return_residual)


# ------------------------------------------------------------------ stores
STORE_BANDS = ["F090W", "F115W", "F150W", "F200W", "F277W", "F356W", "F410M", "F444W"]


def store_header(band, nside, crval, crpix, rot_deg, scale=PIXEL_SCALE, bkg=0.0):
    """A FITS header dict with a TAN WCS: north up to within `rot_deg`, east
    to -x (CD1_1 < 0), `scale` arcsec per pixel."""
    t = np.deg2rad(rot_deg)
    c = scale / 3600.0
    cd = np.array([[-c * np.cos(t), c * np.sin(t)], [c * np.sin(t), c * np.cos(t)]])
    return {"NAXIS": 2, "NAXIS1": int(nside[0]), "NAXIS2": int(nside[1]),
            "CTYPE1": "RA---TAN", "CTYPE2": "DEC--TAN",
            "CRPIX1": float(crpix[0]), "CRPIX2": float(crpix[1]),
            "CRVAL1": float(crval[0]), "CRVAL2": float(crval[1]),
            "CD1_1": float(cd[0, 0]), "CD1_2": float(cd[0, 1]),
            "CD2_1": float(cd[1, 0]), "CD2_2": float(cd[1, 1]),
            "FILTER": band, "BKG": float(bkg)}


def make_store(directory, n_bands=3, exposures_per_band=2, nside=256, super_pixel_size=8,
               seed=0, n_psf=3, n_sources=6, ra0=53.16, dec0=DEC0, rot_deg=20.0,
               mask_frac=0.02, n_locations=2, sip=False):
    """Write a seeded pixel store (HDF5), metadata store (JSON) and PSF store
    (HDF5) in forcepho's layouts into `directory`, and return
    ``dict(pixelstore=, metastore=, psfstore=, bands=, catalog=, epaths=)``.

    Exposures of one band are dithered by up to 10% of the image and rotated
    by up to `rot_deg`; fluxes are a smooth background plus Gaussian noise
    (ierr = 1/sigma, `mask_frac` of pixels with ierr = 0, a few bright pixels
    with signal-to-noise above 100); every header carries a ``BKG`` keyword.
    The catalog holds `n_sources` galaxies near (ra0, dec0)."""
    import json
    import os
    from . import h5lite
    from .fitsio import Header
    from .patches.patch import PSF_COLS
    rng = np.random.default_rng(seed)
    os.makedirs(directory, exist_ok=True)
    nx, ny = (nside, nside) if np.ndim(nside) == 0 else tuple(nside)
    s = super_pixel_size
    bands = STORE_BANDS[:n_bands]
    pix, pattrs, headers, epaths = {}, {}, {}, []
    for b in bands:
        headers[b] = {}
        for j in range(exposures_per_band):
            expID = f"exp{j:02d}"
            shift = rng.uniform(-0.1, 0.1, 2) * np.array([nx, ny]) * PIXEL_SCALE / 3600.0
            crval = (ra0 + shift[0] / np.cos(np.deg2rad(dec0)), dec0 + shift[1])
            crpix = (nx / 2.0 + rng.uniform(-3, 3), ny / 2.0 + rng.uniform(-3, 3))
            bkg = float(rng.normal(0.0, 0.01))
            hdr = store_header(b, (nx, ny), crval, crpix, rng.uniform(-rot_deg, rot_deg), bkg=bkg)
            if sip:
                hdr.update(CTYPE1="RA---TAN-SIP", CTYPE2="DEC--TAN-SIP", A_ORDER=3, B_ORDER=3)
                scale = 4.0 / max(nx, ny) ** 2       # a few pixels at the image edge
                for name in ("A", "B"):
                    for p_, q_ in ((2, 0), (1, 1), (0, 2)):
                        hdr[f"{name}_{p_}_{q_}"] = float(rng.normal(0.0, scale))
                    for p_, q_ in ((3, 0), (2, 1), (1, 2), (0, 3)):
                        hdr[f"{name}_{p_}_{q_}"] = float(rng.normal(0.0, scale / max(nx, ny)))
            xx, yy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
            sky = 0.02 * np.sin(xx / 37.0) * np.cos(yy / 23.0) + bkg
            sigma = 0.05
            im = (sky + rng.normal(0.0, sigma, (nx, ny))).astype(np.float32)
            ierr = np.full((nx, ny), 1.0 / sigma, dtype=np.float32)
            ierr[rng.uniform(size=(nx, ny)) < mask_frac] = 0.0
            hot = rng.uniform(size=(nx, ny)) < 0.001
            im[hot] = 20.0                                   # S/N 400: capped by max_snr=100
            sp = np.concatenate(
                [a.reshape(nx // s, s, ny // s, s).transpose(0, 2, 1, 3).reshape(nx // s, ny // s,
                                                                                s * s)
                 for a in (im, ierr)], axis=-1).astype(np.float32)
            path = f"{b}/{expID}"
            pix[path + "/data"] = sp
            pattrs[path + "/data"] = {"counts_to_flux": 1.0, "flux_units": "image"}
            headers[b][expID] = Header(hdr)
            epaths.append(path)
    pattrs["/"] = {"nside_full": np.array([nx, ny]), "super_pixel_size": np.int64(s)}
    pixelstore = os.path.join(directory, "pixels.h5")
    h5lite.write(pixelstore, pix, pattrs)
    metastore = os.path.join(directory, "meta.json")
    with open(metastore, "w") as f:
        json.dump({b: {e: h.tostring() for e, h in ex.items()} for b, ex in headers.items()}, f)
    # PSF store: n_locations mixtures per band, n_psf Gaussians for each of 9 radius bins
    table = default_table()
    npsf = n_psf * table.n_radii
    psf, psfattrs = {}, {}
    for b in bands:
        par = np.zeros((n_locations, npsf), dtype=PSF_DTYPE)
        for loc in range(n_locations):
            amp = rng.dirichlet(np.ones(n_psf))
            sig = rng.uniform(0.5, 3.0, n_psf)
            for k in range(table.n_radii):
                rows = par[loc, k * n_psf:(k + 1) * n_psf]
                rows["amp"] = amp
                rows["xcen"] = rng.normal(0, 0.05, n_psf)
                rows["ycen"] = rng.normal(0, 0.05, n_psf)
                rows["Cxx"] = sig ** 2
                rows["Cyy"] = sig ** 2 * rng.uniform(0.9, 1.1, n_psf)
                rows["Cxy"] = rng.normal(0, 0.05, n_psf)
                rows["sersic_bin"] = k
        psf[f"{b}/parameters"] = par
        psf[f"{b}/detector_locations"] = rng.uniform(0, nx, (2, n_locations))
        psfattrs[b] = {"n_psf_per_source": np.int64(npsf)}
    psfstore = os.path.join(directory, "psf.h5")
    h5lite.write(psfstore, psf, psfattrs)
    # catalog near the centre, fluxes in every band column
    cols = [(c, np.float64) for c in ["ra", "dec", "q", "pa", "sersic", "rhalf"]]
    cat = np.zeros(n_sources, dtype=cols + [(b, np.float64) for b in bands])
    cosd = np.cos(np.deg2rad(dec0))
    cat["ra"] = ra0 + rng.uniform(-1.0, 1.0, n_sources) / 3600.0 / cosd
    cat["dec"] = dec0 + rng.uniform(-1.0, 1.0, n_sources) / 3600.0
    cat["q"] = rng.uniform(0.5, 0.95, n_sources)
    cat["pa"] = rng.uniform(-1.2, 1.2, n_sources)
    cat["sersic"] = rng.uniform(1.0, 4.0, n_sources)
    cat["rhalf"] = rng.uniform(0.05, 0.3, n_sources)
    for b in bands:
        cat[b] = rng.lognormal(0.0, 0.5, n_sources)
    return dict(pixelstore=pixelstore, metastore=metastore, psfstore=psfstore, bands=bands,
                catalog=cat, epaths=epaths)
