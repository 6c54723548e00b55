"""Pixel, metadata and PSF stores on disk, in forcepho's formats.

Mirrors forcepho/patches/storage.py (``PixelStore``, ``MetaStore``,
``PSFStore``, ``header_to_id``) with the same file layouts, so stores written
by forcepho are read here unchanged:

* pixel store (HDF5): root attributes ``nside_full`` and
  ``super_pixel_size``; one dataset ``<band>/<expID>/data`` per exposure of
  shape ``(nside/s, nside/s, 2 s^2)``: the fluxes of the s x s super-pixel in
  row-major order, then their inverse errors (storage.py:62-300);
* metadata store (JSON): ``{band: {expID: header.tostring()}}``
  (storage.py:303-425);
* PSF store (HDF5): ``<band>/parameters`` of shape (n_locations,
  n_psf_per_source) with fields amp, xcen, ycen, Cxx, Cyy, Cxy, sersic_bin,
  optional ``<band>/detector_locations``, and the ``n_psf_per_source``
  attribute of the band group (storage.py:525-578).

HDF5 goes through :mod:`forcepho_b200.h5lite`, FITS headers through
:mod:`forcepho_b200.fitsio`, and WCSs are :class:`forcepho_b200.wcs.TanWCS`.
"""

import json
import os
from collections import namedtuple

import numpy as np

from .. import h5lite
from ..fitsio import Header
from ..region import polygon_contains
from ..wcs import TanWCS
from .patch import PSF_COLS, PSF_DTYPE

__all__ = ["PixelStore", "MetaStore", "PSFStore", "ImageNameSet", "ImageSet",
           "header_to_id", "PSF_COLS", "PSF_DTYPE"]

ImageNameSet = namedtuple("ImageNames", ["im", "err", "mask", "bkg"])
ImageSet = namedtuple("Images", ["im", "ierr", "mask", "bkg", "hdr", "band", "expID", "names"])

EXP_FMT = "{}/{}"


def header_to_id(hdr, name, framedir=None, split_by_detector=()):
    """(band, expID) of an image: the FILTER keyword (with the detector
    module appended for bands in `split_by_detector`) and the file's base
    name (storage.py:39-57)."""
    filt = hdr["FILTER"]
    if filt in split_by_detector:
        band = f"{filt.upper()}{hdr['DETECTOR'][3].upper()}"
    else:
        band = filt.upper()
    expID = os.path.basename(name).replace(".fits", "")
    if framedir:
        assert framedir in os.path.dirname(name)
        rpath = os.path.dirname(name).replace(framedir, "")
        if rpath.startswith("/"):
            rpath = rpath[1:]
        expID = os.path.join(rpath, expID)
    return band, expID


class PixelStore:
    """Exposures in super-pixel order (see the module docstring).

    Parameters
    ----------
    h5file : path of the HDF5 store; created (with the two attributes) if it
        does not exist.
    nside_full : int or (nx, ny); used only when creating the store.
    super_pixel_size : int, used only when creating the store.
    """

    def __init__(self, h5file, nside_full=2048, super_pixel_size=8, pix_dtype=np.float32):
        self.h5file = h5file
        self.pix_dtype = pix_dtype
        if os.path.exists(h5file):
            with h5lite.File(h5file) as h5:
                self.nside_full = np.asarray(h5.attrs["nside_full"])
                self.super_pixel_size = int(h5.attrs["super_pixel_size"])
        else:
            self.nside_full = np.array(nside_full)
            self.super_pixel_size = int(super_pixel_size)
            h5lite.write(h5file, {}, {"/": {"nside_full": self.nside_full,
                                            "super_pixel_size": np.int64(super_pixel_size)}})
        self.nside_super = self.nside_full / self.super_pixel_size
        self.xpix, self.ypix = self.pixel_coordinates()

    @property
    def imsize(self):
        return (np.zeros(2, dtype=np.int64) + self.nside_full).astype(np.int64)

    def superpixel_corners(self, imsize=None):
        """(nsx, nsy, 4, 2): full-image coordinates of the corner pixels of
        every super-pixel, corners in the order (0,0), (1,0), (1,1), (0,1)
        times (s - 1) from the first pixel (storage.py:117-139)."""
        xpix, ypix = (self.xpix, self.ypix) if imsize is None else self.pixel_coordinates(imsize)
        lower_left = np.array([xpix[:, :, 0], ypix[:, :, 0]])
        offsets = np.array([(0, 0), (1, 0), (1, 1), (0, 1)]) * (self.super_pixel_size - 1)
        corners = offsets[:, :, None, None] + lower_left[None, :, :, :]
        return corners.transpose(2, 3, 0, 1)

    def pixel_coordinates(self, imsize=None):
        """int16 (nsx, nsy, s^2) x and y of every pixel in super-pixel order
        (storage.py:141-149)."""
        imsize = self.imsize if imsize is None else np.asarray(imsize)
        xx, yy = np.meshgrid(np.arange(imsize[0]), np.arange(imsize[1]), indexing="ij")
        packed = self.superpixelize(xx, yy, pix_dtype=np.int64)
        s2 = self.super_pixel_size ** 2
        return packed[:, :, :s2].astype(np.int16), packed[:, :, s2:].astype(np.int16)

    def superpixelize(self, im, ierr, pix_dtype=None):
        """(nsx, nsy, 2 s^2) super-pixel array of an (nx, ny) image and its
        inverse errors: the same element order as the reference's loop
        (storage.py:245-276), by a reshape."""
        s = self.super_pixel_size
        nx, ny = im.shape
        nsx, nsy = nx // s, ny // s
        dt = pix_dtype or self.pix_dtype

        def sp(a):
            return np.asarray(a)[:nsx * s, :nsy * s].reshape(nsx, s, nsy, s) \
                .transpose(0, 2, 1, 3).reshape(nsx, nsy, s * s)
        return np.concatenate([sp(im), sp(ierr)], axis=-1).astype(dt)

    def flux_calibration(self, hdr):
        if "ABMAG" in hdr:
            return 1e9 * 10 ** (0.4 * (8.9 - hdr["ABMAG"])), "nJy"
        return 1.0, "counts"

    def add_exposure(self, imset, bitmask=None, do_fluxcal=False):
        """Background-subtract, mask, optionally flux-calibrate and
        super-pixelize one exposure and write it as ``band/expID/data``
        (storage.py:151-243; an existing dataset of that path is replaced).
        The whole file is rewritten (see write_exposures)."""
        band, expID, hdr = imset.band, imset.expID, imset.hdr
        im = np.array(imset.im, dtype=np.float64 if np.asarray(imset.im).dtype == np.float64
                      else np.float32)
        ierr = np.array(imset.ierr, dtype=im.dtype)
        bkg = np.zeros_like(im) if imset.bkg is None else np.asarray(imset.bkg)
        if imset.bkg is not None:
            im -= bkg
        mask = ~(np.isfinite(ierr) & np.isfinite(im) & (ierr >= 0))
        if imset.mask is not None:
            pmask = np.asarray(imset.mask)
            if bitmask:
                pmask = np.bitwise_and(pmask, bitmask) != 0
            mask = mask | pmask
        ierr[mask] = 0
        im[mask] = 0
        gb = np.isfinite(bkg)
        im[mask & gb] = bkg[mask & gb]
        if do_fluxcal:
            fluxconv, unitname = self.flux_calibration(hdr)
            im *= fluxconv
            ierr *= 1.0 / fluxconv
        else:
            fluxconv, unitname = 1.0, "image"
        imsize = np.array(im.shape)
        assert np.all(np.mod(imsize, self.super_pixel_size) == 0)
        if np.any(imsize != self.imsize):
            raise ValueError("Image is not the expected size")
        superpixels = self.superpixelize(im, ierr)
        assert np.all(np.isfinite(superpixels)), f"non-finite pixels in exposure {expID}"
        attrs = {"counts_to_flux": fluxconv, "flux_units": unitname}
        if bitmask:
            attrs["bitmask_applied"] = bitmask
        if isinstance(imset.names, str):
            attrs["image_name"] = imset.names
        elif imset.names is not None:
            for f, v in zip(imset.names._fields, imset.names):
                if isinstance(v, str):
                    attrs[f] = v
        self.write_exposures({EXP_FMT.format(band, expID): (superpixels, attrs)})

    def write_exposures(self, exposures):
        """Add or replace exposures: {"band/expID": (superpixels, attrs)}.
        The file is rewritten; existing exposures are streamed from a memory
        map of the old file, so memory use does not grow with the store."""
        self.close()
        data, attrs = h5lite.read_tree(self.h5file, memmap=True)
        for path, (sp, at) in exposures.items():
            data[path + "/data"] = np.asarray(sp, dtype=self.pix_dtype)
            attrs[path + "/data"] = dict(at)
        h5lite.write(self.h5file, data, attrs)

    def exposure_paths(self):
        """["band/expID", ...] in file order (bands, then exposures, sorted)."""
        h5 = self.data
        return [f"{b}/{e}" for b in h5.keys() for e in h5[b].keys()]

    @property
    def data(self):
        try:
            return self._read_handle
        except AttributeError:
            self._read_handle = h5lite.File(self.h5file)
            return self._read_handle

    def close(self):
        try:
            self._read_handle.close()
            del self._read_handle
        except AttributeError:
            pass


class MetaStore:
    """FITS headers (and TAN WCSs) of the exposures, keyed by band then
    expID (storage.py:303-510)."""

    def __init__(self, metastorefile=None, use_gwcs=False, load_all=False):
        self.headers, self.wcs = {}, {}
        if use_gwcs:
            raise NotImplementedError("gWCS is not supported")
        if metastorefile is not None:
            self.headers = self.read_from_file(metastorefile)
            if load_all:
                self.populate_wcs()

    def populate_wcs(self, gwcs_file=None):
        self.wcs = {band: {e: TanWCS(h) for e, h in exps.items()}
                    for band, exps in self.headers.items()}

    def get_wcs(self, band, expID):
        w = self.wcs.setdefault(band, {})
        if expID not in w:
            w[expID] = TanWCS(self.headers[band][expID])
        return w[expID]

    def add_exposure(self, imset):
        self.headers.setdefault(imset.band, {})[imset.expID] = imset.hdr

    def write_to_file(self, filename):
        assert ".json" in filename
        out = {b: {e: (h.tostring() if hasattr(h, "tostring") else Header(h).tostring())
                   for e, h in exps.items()} for b, exps in self.headers.items()}
        with open(filename, "w") as f:
            json.dump(out, f)

    def read_from_file(self, filename):
        with open(filename, "r") as f:
            s = json.load(f)
        return {b: {e: Header.fromstring(h) for e, h in exps.items()} for b, exps in s.items()}

    def find_exposures(self, sky, bandlist):
        """(expIDs, bands) of the exposures whose footprint contains `sky`
        (storage.py:427-490): an optional rough S_REGION test, then the
        image corners mapped to the sky."""
        epaths, bands = [], []
        for band in bandlist:
            if band not in self.headers:
                continue
            for expID, hdr in self.headers[band].items():
                try:
                    polys = str(hdr["S_REGION"]).split()[2:]
                    rough = np.array([float(p) for p in polys]).reshape(4, 2)
                    if not polygon_contains(rough, np.atleast_2d(sky))[0]:
                        continue
                except KeyError:
                    pass
                wcs = self.get_wcs(band, expID)
                nx, ny = hdr["NAXIS1"], hdr["NAXIS2"]
                bbox = np.array([[0, 0], [0, ny], [nx, nx], [nx, 0]]).T
                bbox = np.array(wcs.pixel_to_world_values(bbox[0], bbox[1])).T
                if polygon_contains(bbox, np.atleast_2d(sky))[0]:
                    epaths.append(expID)
                    bands.append(band)
        return epaths, bands

    @property
    def nexp(self):
        return sum(len(e) for e in self.headers.values())


class PSFStore:
    """PSF Gaussian mixtures per band (storage.py:525-578)."""

    def __init__(self, h5file):
        self.h5file = h5file
        self._rows = {}      # (band, location) -> rows, read once
        self._locs = {}

    def lookup(self, band, xy=None):
        """(n_psf_per_source,) PSF rows of `band`: the detector location
        nearest to `xy` if the band has locations and `xy` is given, else
        the first.  Rows are read from the file once per (band, location)."""
        choose = 0
        if xy is not None:
            if band not in self._locs:
                g = self.data[band]
                self._locs[band] = (np.asarray(g["detector_locations"][:])
                                    if "detector_locations" in g else None)
            locs = self._locs[band]
            if locs is not None:
                xp, yp = locs
                choose = int(np.hypot(xy[0] - xp, xy[1] - yp).argmin())
        key = (band, choose)
        if key not in self._rows:
            self._rows[key] = _as_psf_rows(self.data[band]["parameters"][choose])
        return self._rows[key].copy()

    def get_local_psf(self, band="F090W", source=None, wcs=None):
        xy = wcs.world_to_pixel_values(source.ra, source.dec) if wcs is not None else None
        return self.lookup(band, xy=xy)

    def n_psf_per_source(self, band):
        key = ("npsf", band)
        if key not in self._rows:
            self._rows[key] = int(self.data[band].attrs["n_psf_per_source"])
        return self._rows[key]

    @property
    def data(self):
        try:
            return self._h5
        except AttributeError:
            self._h5 = h5lite.File(self.h5file)
            return self._h5


def _as_psf_rows(p):
    """PSF rows in PSF_DTYPE from either field layout forcepho stores use:
    named columns, or ``gauss_params`` (6) + ``sersic_bin``."""
    p = np.asarray(p)
    out = np.zeros(p.shape, dtype=PSF_DTYPE)
    if "gauss_params" in p.dtype.names:
        for i, c in enumerate(PSF_COLS):
            out[c] = p["gauss_params"][..., i]
    else:
        for c in PSF_COLS:
            out[c] = p[c]
    out["sersic_bin"] = p["sersic_bin"]
    return out
