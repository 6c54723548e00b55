"""Patches packed from exposures on disk or in memory.

Mirrors forcepho/patches/pixel_patch.py: :class:`PixelPatch` finds the
exposures of a region and packs their pixels (``pack_pix``: per exposure, the
selected pixels concatenated band by band, with ``exposure_start/N`` and
``band_start/N``; optional background offsets and a cap on the
signal-to-noise ratio), and the three sources of pixels:

* :class:`StorePatch` -- a super-pixel :class:`~.storage.PixelStore` and its
  :class:`~.storage.MetaStore` (super-pixels with a corner in the region);
* :class:`FITSPatch` -- FITS images and uncertainty maps (pixels with a
  corner in the region, padded to a multiple of ``warp_size`` with
  ``ierr = 0`` and ``x = y = -1``);
* :class:`DirectPatch` -- arrays given in dictionaries.

:class:`forcepho_b200.patches.device_store.GPUStorePatch` does the
``StorePatch`` selection and packing with CUDA kernels on exposures held in
GPU memory.
"""

import numpy as np

from .. import fitsio
from ..wcs import TanWCS
from .patch import Patch
from .storage import MetaStore, PixelStore

__all__ = ["PixelPatch", "StorePatch", "FITSPatch", "DirectPatch", "JWST_BANDS"]

JWST_BANDS = ["F090W", "F115W", "F150W", "F200W", "F277W", "F335M", "F356W", "F410M", "F444W"]


class PixelPatch(Patch):
    """Packing of pixel data from lists of exposures; subclasses implement
    :meth:`find_exposures` and :meth:`find_pixels`
    (forcepho/patches/pixel_patch.py:23-214)."""

    def __init__(self, psfstore="", splinedata="", spline_smoothing=None, return_residual=False,
                 meta_dtype=np.float32, pix_dtype=np.float32, debug=0):
        super().__init__(psfstore=psfstore, splinedata=splinedata,
                         spline_smoothing=spline_smoothing, return_residual=return_residual,
                         meta_dtype=meta_dtype, pix_dtype=pix_dtype, debug=debug)
        self.background_offsets = None
        self.max_snr = None

    def build_patch(self, region=None, sourcecat=None, allbands=JWST_BANDS,
                    tweak_background=False):
        """Find the exposures of `region`, pack their pixels and, if a
        source catalog is given, the scene metadata."""
        self.hdrs, self.wcses, self.epaths, self.bands = self.find_exposures(region, allbands)
        if len(self.epaths) == 0:
            raise ValueError("No exposures in the specified bands overlap the region")
        if tweak_background:
            self.background_offsets = [hdr.get(tweak_background, 0.0) for hdr in self.hdrs]
        else:
            self.background_offsets = None
        self._set_band_index(allbands)
        self.pack_pix(region=region)
        if sourcecat is not None:
            self.pack_meta(self.set_scene(sourcecat))
        self._dirty_data = False

    def _set_band_index(self, allbands):
        allbands = list(allbands)
        band_ids = [allbands.index(b) for b in self.bands]
        assert (np.diff(band_ids) >= 0).all(), "Exposures must be sorted by band"
        u, n = np.unique(band_ids, return_counts=True)
        self.uniq_bands, self.n_exp_per_band = u, n
        self.bandlist = [allbands[i] for i in self.uniq_bands]

    def pack_pix(self, region, dtype=None):
        """Concatenate the exposures' pixels and fill the index arrays
        (pixel_patch.py:124-198)."""
        nb, ne = len(self.uniq_bands), len(self.epaths)
        self.band_start = np.empty(nb, dtype=np.int16)
        self.band_N = np.zeros(nb, dtype=np.int16)
        self.exposure_start = np.empty(ne, dtype=np.int32)
        self.exposure_N = np.empty(ne, dtype=np.int32)
        data, ierr, xpix, ypix = [], [], [], []
        b, i = 0, 0
        for e, wcs in enumerate(self.wcses):
            pixdat = self.find_pixels(self.epaths[e], wcs, region)
            n_pix = pixdat[0].size
            assert n_pix > 0, f"There were no valid pixels in exposure {self.epaths[e]}"
            if self.debug > 0:
                assert np.all(np.isfinite(pixdat[0] * pixdat[1])), \
                    f"There were non-finite pixels in exposure {self.epaths[e]}"
            fluxes = pixdat[0]
            if self.background_offsets is not None:
                fluxes = pixdat[0] - self.background_offsets[e]
            if e > 0 and self.bands[e] != self.bands[e - 1]:
                b += 1
            self.band_N[b] += 1
            self.exposure_start[e] = i
            self.exposure_N[e] = n_pix
            data.append(fluxes)
            ierr.append(pixdat[1])
            xpix.append(pixdat[2])
            ypix.append(pixdat[3])
            i += n_pix
        self.data = np.concatenate([np.reshape(a, -1) for a in data]).astype(np.float32)
        self.ierr = np.concatenate([np.reshape(a, -1) for a in ierr]).astype(np.float32)
        self.xpix = np.concatenate([np.reshape(a, -1) for a in xpix]).astype(np.float32)
        self.ypix = np.concatenate([np.reshape(a, -1) for a in ypix]).astype(np.float32)
        self.band_start[0] = 0
        self.band_start[1:] = np.cumsum(self.band_N)[:-1]
        if getattr(self, "max_snr", None):
            self._cap_snr(max_snr=self.max_snr)

    def _cap_snr(self, max_snr=None):
        if max_snr:
            to_cap = (self.ierr > 0) & (self.data * self.ierr > max_snr)
            self.ierr[to_cap] = max_snr / self.data[to_cap]

    def find_exposures(self, region, bandlist):
        raise NotImplementedError

    def find_pixels(self, epath, wcs, region):
        raise NotImplementedError


class StorePatch(PixelPatch):
    """Pixels from a super-pixel pixel store and headers from a metadata
    store (pixel_patch.py:216-342)."""

    def __init__(self, pixelstore="", metastore="", psfstore="", splinedata="",
                 spline_smoothing=None, return_residual=False, meta_dtype=np.float32,
                 pix_dtype=np.float32, debug=0):
        super().__init__(psfstore=psfstore, splinedata=splinedata,
                         spline_smoothing=spline_smoothing, return_residual=return_residual,
                         meta_dtype=meta_dtype, pix_dtype=pix_dtype, debug=debug)
        self.metastore = MetaStore(metastore) if isinstance(metastore, str) else metastore
        self.pixelstore = PixelStore(pixelstore) if isinstance(pixelstore, str) else pixelstore

    def find_exposures(self, region, bandlist):
        """Exposures with a corner of the region's bounding box inside the
        image and at least one super-pixel in the region, in `bandlist`
        order then metadata-store order."""
        imsize = np.zeros(2) + self.pixelstore.nside_full
        corners = self.pixelstore.superpixel_corners()
        bra, bdec = region.bounding_box
        epaths, bands, hdrs, wcses = [], [], [], []
        for band in bandlist:
            if band not in self.metastore.headers:
                continue
            for expID in self.metastore.headers[band].keys():
                wcs = self.metastore.get_wcs(band, expID)
                bx, by = wcs.world_to_pixel_values(bra, bdec)
                if not np.any((bx > 0) & (bx < imsize[0]) & (by > 0) & (by < imsize[1])):
                    continue
                sx, sy = region.contains(corners[..., 0], corners[..., 1], wcs)
                if len(sx) == 0:
                    continue
                wcses.append(wcs)
                epaths.append(f"{band}/{expID}")
                bands.append(band)
                hdrs.append(self.metastore.headers[band][expID])
        return hdrs, wcses, epaths, bands

    def find_pixels(self, epath, wcs, region):
        """(data, ierr, xpix, ypix) of the super-pixels in the region, each of
        shape (n_superpixels, s^2), in row-major super-pixel order."""
        s2 = self.pixelstore.super_pixel_size ** 2
        corners = self.pixelstore.superpixel_corners()
        sx, sy = region.contains(corners[..., 0], corners[..., 1], wcs)
        sp = self.pixelstore.data[epath + "/data"].array()[sx, sy, :]
        return (sp[:, :s2], sp[:, s2:], self.pixelstore.xpix[sx, sy, :],
                self.pixelstore.ypix[sx, sy, :])


class FITSPatch(PixelPatch):
    """Pixels from FITS images and uncertainty maps (pixel_patch.py:345-482).

    ``sci_ext`` and ``unc_ext`` are extension names (EXTNAME) or indices.
    """

    def __init__(self, fitsfiles="", psfstore="", splinedata="", spline_smoothing=None,
                 return_residual=False, sci_ext="SCI", unc_ext="ERR", meta_dtype=np.float32,
                 pix_dtype=np.float32, debug=0):
        super().__init__(psfstore=psfstore, splinedata=splinedata,
                         spline_smoothing=spline_smoothing, return_residual=return_residual,
                         meta_dtype=meta_dtype, pix_dtype=pix_dtype, debug=debug)
        self.fitsfiles = fitsfiles
        self.sci_ext, self.unc_ext = sci_ext, unc_ext
        self.snr = None
        self.unc = None
        self.warp_size = 64

    def find_exposures(self, region, bandlist, do_check=True):
        fitsfiles = np.atleast_1d(np.array(self.fitsfiles))
        hdrs_all = [fitsio.getheader(f, self.sci_ext) for f in fitsfiles]
        imbands = np.array([str(h["FILTER"]).strip() for h in hdrs_all])
        epaths, bands, hdrs, wcses = [], [], [], []
        for band in bandlist:
            for i in np.flatnonzero(imbands == band):
                hdr = hdrs_all[i]
                wcs = TanWCS(hdr)
                if region is not None and do_check:
                    bra, bdec = region.bounding_box
                    nx, ny = hdr["NAXIS1"], hdr["NAXIS2"]
                    bx, by = wcs.world_to_pixel_values(bra, bdec)
                    inim = np.any((bx > 0) & (bx < nx) & (by > 0) & (by < ny))
                    around = ((nx < bx.max()) & (bx.min() < 0) & (ny < by.max()) & (by.min() < 0))
                    if not (inim | around):
                        continue
                epaths.append(str(fitsfiles[i]))
                wcses.append(wcs)
                bands.append(imbands[i])
                hdrs.append(hdr)
        return hdrs, wcses, epaths, bands

    def find_pixels(self, epath, wcs, region):
        flux = np.array(fitsio.getdata(epath, self.sci_ext).T)
        if getattr(self, "snr", None) is not None:
            ie = self.snr / flux
        elif getattr(self, "unc", None) is not None:
            ie = np.zeros_like(flux) + 1.0 / self.unc
        else:
            with np.errstate(divide="ignore"):
                ie = 1.0 / fitsio.getdata(epath, self.unc_ext).T
        bad = ~np.isfinite(flux) | ~np.isfinite(ie) | (ie < 0)
        ie = np.array(ie)
        ie[bad] = 0
        flux[bad] = 0
        nx, ny = flux.shape
        yp, xp = np.meshgrid(np.arange(ny), np.arange(nx))
        if region is None:
            sx, sy = slice(None), slice(None)
        else:
            offsets = np.array([(0, 0), (1, 0), (1, 1), (0, 1)])
            lower_left = np.array([xp, yp])
            corners = (offsets[:, :, None, None] + lower_left[None]).transpose(2, 3, 0, 1)
            sx, sy = region.contains(corners[..., 0], corners[..., 1], wcs)
        flux, ie = flux[sx, sy].reshape(-1), ie[sx, sy].reshape(-1)
        xp, yp = xp[sx, sy].reshape(-1), yp[sx, sy].reshape(-1)
        warp = getattr(self, "warp_size", 64)
        pad = warp - np.mod(len(flux), warp)
        if pad != warp:
            ie = np.append(ie, np.zeros(pad, dtype=ie.dtype))
            flux = np.append(flux, np.zeros(pad, dtype=flux.dtype))
            xp = np.append(xp, np.zeros(pad, dtype=xp.dtype) - 1)
            yp = np.append(yp, np.zeros(pad, dtype=yp.dtype) - 1)
        return flux, ie, xp, yp


class DirectPatch(PixelPatch):
    """Pixels given directly: ``pixel_dict[epath]`` with ``flux``, ``ierr``,
    ``xpix``, ``ypix`` arrays and ``header_dict[epath]`` with FILTER and a
    TAN WCS (pixel_patch.py:485-550)."""

    def __init__(self, pixel_dict=None, header_dict=None, psfstore="", splinedata="",
                 spline_smoothing=None, return_residual=False, meta_dtype=np.float32,
                 pix_dtype=np.float32, debug=0):
        super().__init__(psfstore=psfstore, splinedata=splinedata,
                         spline_smoothing=spline_smoothing, return_residual=return_residual,
                         meta_dtype=meta_dtype, pix_dtype=pix_dtype, debug=debug)
        self.pixel_dict = pixel_dict or {}
        self.header_dict = header_dict or {}
        self.snr = None
        self.unc = None

    def find_exposures(self, region, bandlist, do_check=True):
        epaths = list(self.header_dict.keys())
        hdrs = [self.header_dict[e] for e in epaths]
        return hdrs, [TanWCS(h) for h in hdrs], epaths, [str(h["FILTER"]).strip() for h in hdrs]

    def find_pixels(self, epath, wcs, region):
        p = self.pixel_dict[epath]
        return p["flux"], p["ierr"], p["xpix"], p["ypix"]
