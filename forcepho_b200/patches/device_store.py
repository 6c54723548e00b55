"""Exposures held in GPU memory, and patches packed from them on the device.

The reference packs every patch on the host: it reads each overlapping
exposure's whole super-pixel array from the HDF5 pixel store, tests every
super-pixel's corners against the region with numpy, and concatenates the
selected pixels before copying them to the GPU
(forcepho/patches/pixel_patch.py:124-198, 297-342).  When patches are fit
one after another that work repeats for every patch.

:class:`DeviceStore` uploads the exposures once (the ``fpho_store`` of the C
ABI: 32 MiB per 2048x2048 exposure, so a B200 holds thousands) and
:class:`GPUStorePatch` -- a :class:`~.pixel_patch.StorePatch` with the GPU
mix-in -- selects super-pixels and packs the patch's pixel arrays with CUDA
kernels straight into device memory, in the reference's order, so the host
keeps only the index arrays and the per-scene metadata.
"""

import ctypes

import numpy as np

from .. import _lib
from ..region import REGION_CIRCLE, REGION_RECT, CircularRegion
from ..wcs import TanWCSStack
from .device_patch import DevicePatch, GPUPatchMixin
from .pixel_patch import StorePatch

__all__ = ["DeviceStore", "GPUStorePatch", "REGION_DTYPE", "region_records"]

# fpho_region of include/fpho.h
REGION_DTYPE = np.dtype([("kind", np.int32), ("reserved", np.int32), ("p", np.float64, 14)])


def region_records(region, wcses, stack=None):
    """One ``fpho_region`` record per exposure WCS.  A circle's centre and
    radius are mapped to every exposure's pixels in one numpy pass over
    `stack` (a :class:`~forcepho_b200.wcs.TanWCSStack` of `wcses`, built if
    not given), with the arithmetic of ``CircularRegion.pixel_circle``."""
    out = np.zeros(len(wcses), dtype=REGION_DTYPE)
    if len(wcses) == 0:
        return out
    if isinstance(region, CircularRegion):
        stack = stack if stack is not None else TanWCSStack(wcses)
        x, y = stack.world_to_pixel_values([region.ra, region.ra],
                                           [region.dec, region.dec + region.radius])
        xc, yc, xr, yr = x[:, 0], y[:, 0], x[:, 1], y[:, 1]
        out["kind"] = REGION_CIRCLE
        out["p"][:, 0], out["p"][:, 1] = xc, yc
        out["p"][:, 2] = (xc - xr) ** 2 + (yc - yr) ** 2
        return out
    for i, w in enumerate(wcses):
        kind, p = region.device_params(w)
        if kind not in (REGION_CIRCLE, REGION_RECT):
            raise ValueError(f"region kind {kind}")
        out[i]["kind"] = kind
        out[i]["p"][:len(p)] = p
    return out


class DeviceStore:
    """Super-pixel exposures resident in GPU memory.

    Parameters
    ----------
    nside : int or (nx, ny), image size in pixels
    super_pixel_size : int
    max_exposures : capacity (all device memory is allocated here)
    """

    def __init__(self, nside, super_pixel_size=8, max_exposures=64):
        nx, ny = (int(nside), int(nside)) if np.ndim(nside) == 0 else (int(nside[0]),
                                                                       int(nside[1]))
        h = ctypes.c_void_p()
        _lib.call("fpho_store_create", nx, ny, int(super_pixel_size), int(max_exposures),
                  ctypes.byref(h))
        self.handle = h.value
        self.nside = (nx, ny)
        self.super_pixel_size = int(super_pixel_size)
        self.names = []

    @classmethod
    def from_pixelstore(cls, pixelstore, paths=None, max_exposures=None):
        """Upload exposures (``"band/expID"`` paths; default all) of a
        :class:`~.storage.PixelStore`."""
        paths = list(paths) if paths is not None else pixelstore.exposure_paths()
        st = cls(pixelstore.imsize, pixelstore.super_pixel_size,
                 max_exposures or max(len(paths), 1))
        for p in paths:
            st.add(pixelstore.data[p + "/data"].array(), name=p)
        return st

    def add(self, superpixels, name=None, stream=None):
        """Append one exposure: an (nsx, nsy, 2 s^2) float32 array on the host
        or a CUDA tensor of that shape.  Returns its index."""
        nsx, nsy = self.nside[0] // self.super_pixel_size, self.nside[1] // self.super_pixel_size
        shape = (nsx, nsy, 2 * self.super_pixel_size ** 2)
        idx = ctypes.c_int()
        if hasattr(superpixels, "is_cuda") and superpixels.is_cuda:
            import torch
            t = superpixels.contiguous().to(torch.float32)
            if tuple(t.shape) != shape:
                raise ValueError(f"super-pixel array of shape {tuple(t.shape)}, expected {shape}")
            _lib.call("fpho_store_add_exposure", self.handle, t.data_ptr(), 1, stream,
                      ctypes.byref(idx))
            if stream is None:
                torch.cuda.synchronize()
        else:
            a = np.ascontiguousarray(superpixels, dtype=np.float32)
            if a.shape != shape:
                raise ValueError(f"super-pixel array of shape {a.shape}, expected {shape}")
            _lib.call("fpho_store_add_exposure", self.handle, a.ctypes.data, 0, stream,
                      ctypes.byref(idx))
        self.names.append(name if name is not None else str(idx.value))
        return idx.value

    def index(self, name):
        return self.names.index(name)

    def info(self):
        out = (ctypes.c_int64 * 6)()
        _lib.call("fpho_store_info", self.handle, out)
        return dict(zip(["nsx", "nsy", "super_pixel_size", "n_exposures", "capacity",
                         "bytes_per_exposure"], list(out)))

    def count(self, indices, regions, stream=None):
        """Selected super-pixels of each exposure (`regions`: REGION_DTYPE
        records, one per index)."""
        idx = np.ascontiguousarray(indices, dtype=np.int32)
        reg = np.ascontiguousarray(regions, dtype=REGION_DTYPE)
        out = np.zeros(len(idx), dtype=np.int32)
        _lib.call("fpho_store_count", self.handle, len(idx), idx.ctypes.data, reg.ctypes.data,
                  out.ctypes.data, stream)
        return out

    def gather(self, indices, regions, background=None, max_snr=None, npix=None, stream=None):
        """Pack the selected pixels: returns (data, ierr, xpix, ypix) float32
        CUDA tensors and the exposure_start, exposure_N arrays."""
        import torch
        idx = np.ascontiguousarray(indices, dtype=np.int32)
        reg = np.ascontiguousarray(regions, dtype=REGION_DTYPE)
        if npix is None:
            npix = int(self.count(idx, reg, stream).astype(np.int64).sum()) \
                * self.super_pixel_size ** 2
        bufs = [torch.empty(max(npix, 1), dtype=torch.float32, device="cuda") for _ in range(4)]
        bg = None if background is None else np.ascontiguousarray(background, dtype=np.float32)
        start = np.zeros(len(idx), dtype=np.int32)
        n = np.zeros(len(idx), dtype=np.int32)
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        _lib.call("fpho_store_gather", self.handle, len(idx), idx.ctypes.data, reg.ctypes.data,
                  None if bg is None else bg.ctypes.data, float(max_snr or 0.0),
                  *[b.data_ptr() for b in bufs], int(npix), start.ctypes.data, n.ctypes.data,
                  stream)
        total = int(n.astype(np.int64).sum())
        return [b[:total] for b in bufs], start, n

    def gather_many(self, groups, max_snr=None, stream=None):
        """Pack several patches in one count and one gather call.  `groups`
        is a list of (indices, regions, background-or-None), one per patch;
        returns, per patch, ((data, ierr, xpix, ypix) views of one shared
        buffer, exposure_start relative to the patch, exposure_N)."""
        if not groups:
            return []
        idx = np.concatenate([np.asarray(g[0], dtype=np.int32) for g in groups])
        recs = np.concatenate([np.asarray(g[1], dtype=REGION_DTYPE) for g in groups])
        bg = None
        if any(g[2] is not None for g in groups):
            bg = np.concatenate([np.zeros(len(g[0]), np.float32) if g[2] is None
                                 else np.asarray(g[2], dtype=np.float32) for g in groups])
        pix, start, n = self.gather(idx, recs, background=bg, max_snr=max_snr, stream=stream)
        out, e0 = [], 0
        for g in groups:
            e1 = e0 + len(g[0])
            p0 = int(start[e0]) if e1 > e0 else 0
            p1 = p0 + int(np.asarray(n[e0:e1], dtype=np.int64).sum())
            out.append(([t[p0:p1] for t in pix], (start[e0:e1] - p0).astype(np.int32),
                        n[e0:e1].copy()))
            e0 = e1
        return out

    def time_gather(self, enable=True):
        """Time the gather kernel of every following :meth:`gather` with CUDA
        events; :meth:`last_gather_ms` reads the last one."""
        _lib.call("fpho_store_time_gather", self.handle, int(bool(enable)))

    def last_gather_ms(self):
        ms = ctypes.c_float()
        _lib.call("fpho_store_last_gather_ms", self.handle, ctypes.byref(ms))
        return ms.value

    def free(self):
        if getattr(self, "handle", None):
            _lib.lib.fpho_store_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GPUStorePatch(StorePatch, GPUPatchMixin):
    """A :class:`~.pixel_patch.StorePatch` whose super-pixel selection and
    pixel packing run on the GPU over a :class:`DeviceStore`.

    The exposures found and the packed arrays are those of the host
    ``StorePatch`` (bounding-box corner check on the host, then exposures with
    at least one super-pixel in the region).  The pixel arrays stay on the
    device (``pixels``: data, ierr, xpix, ypix tensors);
    :meth:`pixels_to_host` copies them into the usual attributes.

    Parameters are those of ``StorePatch`` plus ``device_store`` (default:
    upload every exposure of the pixel store).
    """

    def __init__(self, pixelstore="", metastore="", psfstore="", splinedata="",
                 spline_smoothing=None, return_residual=False, device_store=None, debug=0):
        super().__init__(pixelstore=pixelstore, metastore=metastore, psfstore=psfstore,
                         splinedata=splinedata, spline_smoothing=spline_smoothing,
                         return_residual=return_residual, debug=debug)
        self.device_store = device_store or DeviceStore.from_pixelstore(self.pixelstore)
        self.pixels = None
        self.device_patch = None

    def _exposure_table(self, bandlist):
        """(band, expID, wcs, store index) of every exposure of `bandlist`
        in metadata-store order, and their WCS stack (cached)."""
        key = tuple(bandlist)
        if getattr(self, "_exp_table_key", None) != key:
            rows = [(b, e, self.metastore.get_wcs(b, e), self.device_store.index(f"{b}/{e}"))
                    for b in bandlist if b in self.metastore.headers
                    for e in self.metastore.headers[b].keys()]
            self._exp_table = (rows, TanWCSStack([r[2] for r in rows]) if rows else None)
            self._exp_table_key = key
        return self._exp_table

    def find_exposures(self, region, bandlist):
        """As StorePatch.find_exposures: a corner of the region's bounding
        box inside the image (all exposures in one numpy pass), then at least
        one super-pixel in the region (the count kernel)."""
        rows, stack = self._exposure_table(bandlist)
        self._records = {}
        if not rows:
            return [], [], [], []
        imsize = np.zeros(2) + self.pixelstore.nside_full
        bra, bdec = region.bounding_box
        bx, by = stack.world_to_pixel_values(bra, bdec)
        inim = np.any((bx > 0) & (bx < imsize[0]) & (by > 0) & (by < imsize[1]), axis=1)
        sel = np.flatnonzero(inim)
        if len(sel) == 0:
            return [], [], [], []
        recs = region_records(region, [rows[i][2] for i in range(len(rows))], stack)[sel]
        counts = self.device_store.count([rows[i][3] for i in sel], recs)
        keep = [(rows[i], rec, n) for i, rec, n in zip(sel, recs, counts) if n > 0]
        self._records = {f"{r[0]}/{r[1]}": (rec, int(n)) for r, rec, n in keep}
        keep = [(r, rec) for r, rec, _ in keep]
        return ([self.metastore.headers[r[0]][r[1]] for r, _ in keep], [r[2] for r, _ in keep],
                [f"{r[0]}/{r[1]}" for r, _ in keep], [r[0] for r, _ in keep])

    def pack_pix(self, region, dtype=None):
        idx = [self.device_store.index(p) for p in self.epaths]
        cached = getattr(self, "_records", {})
        npix = None
        if all(p in cached for p in self.epaths):     # from find_exposures: no second count
            regs = np.array([cached[p][0] for p in self.epaths], dtype=REGION_DTYPE)
            npix = sum(cached[p][1] for p in self.epaths) * self.device_store.super_pixel_size ** 2
        else:
            regs = region_records(region, self.wcses)
        pix, start, n = self.device_store.gather(idx, regs, background=self.background_offsets,
                                                 max_snr=getattr(self, "max_snr", None),
                                                 npix=npix)
        self._install_pixels(pix, start, n)

    def build_patches(self, regions, sourcecats=None, allbands=None, tweak_background=False):
        """Build one patch per region with a single count and a single gather
        over all of them (the copy kernel then moves every patch's pixels in
        one launch).  Returns new GPUStorePatch objects sharing this one's
        stores; each holds the same arrays ``build_patch`` gives for its
        region.  `sourcecats`: one catalog per region, or None."""
        import copy
        allbands = list(allbands) if allbands is not None else list(self.metastore.headers)
        rows, stack = self._exposure_table(allbands)
        imsize = np.zeros(2) + self.pixelstore.nside_full
        cands = []
        for region in regions:
            if not rows:
                cands.append(([], None))
                continue
            bra, bdec = region.bounding_box
            bx, by = stack.world_to_pixel_values(bra, bdec)
            sel = np.flatnonzero(np.any((bx > 0) & (bx < imsize[0]) & (by > 0) &
                                        (by < imsize[1]), axis=1))
            recs = region_records(region, [r[2] for r in rows], stack)[sel]
            cands.append((sel, recs))
        all_idx = [rows[i][3] for sel, _ in cands for i in sel]
        all_recs = [rec for sel, recs in cands if len(sel) for rec in recs]
        counts = (self.device_store.count(all_idx, np.array(all_recs, dtype=REGION_DTYPE))
                  if all_idx else np.zeros(0, np.int32))
        patches, groups, k = [], [], 0
        for (sel, recs), region in zip(cands, regions):
            cnt = counts[k:k + len(sel)]
            k += len(sel)
            keep = [(rows[i], rec) for i, rec, c in zip(sel, recs if recs is not None else [],
                                                          cnt) if c > 0]
            if not keep:
                raise ValueError("No exposures in the specified bands overlap the region")
            p = copy.copy(self)
            p.pixels, p.device_patch, p._records = None, None, {}
            p.hdrs = [self.metastore.headers[r[0]][r[1]] for r, _ in keep]
            p.wcses = [r[2] for r, _ in keep]
            p.epaths = [f"{r[0]}/{r[1]}" for r, _ in keep]
            p.bands = [r[0] for r, _ in keep]
            p.background_offsets = ([h.get(tweak_background, 0.0) for h in p.hdrs]
                                    if tweak_background else None)
            p._set_band_index(allbands)
            patches.append(p)
            groups.append(([r[3] for r, _ in keep],
                           np.array([rec for _, rec in keep], dtype=REGION_DTYPE),
                           p.background_offsets))
        packed = self.device_store.gather_many(groups, max_snr=getattr(self, "max_snr", None))
        for i, (p, (pix, start, n)) in enumerate(zip(patches, packed)):
            p._install_pixels(pix, start, n)
            if sourcecats is not None:
                p.pack_meta(p.set_scene(sourcecats[i]))
            p._dirty_data = False
        return patches

    def _install_pixels(self, pix, start, n):
        self.pixels = dict(zip(["data", "ierr", "xpix", "ypix"], pix))
        for k in ("data", "ierr", "xpix", "ypix"):
            self.__dict__.pop(k, None)
        self.exposure_start, self.exposure_N = start, n
        nb = len(self.uniq_bands)
        self.band_N = np.zeros(nb, dtype=np.int16)
        b = 0
        for e in range(len(self.epaths)):
            if e > 0 and self.bands[e] != self.bands[e - 1]:
                b += 1
            self.band_N[b] += 1
        self.band_start = np.zeros(nb, dtype=np.int16)
        self.band_start[1:] = np.cumsum(self.band_N)[:-1]

    @property
    def npix(self):
        return int(np.asarray(self.exposure_N, dtype=np.int64).sum())

    def host_struct(self, residual=None, pointers=None):
        """As PatchBase.host_struct, with the pixel fields pointing at the
        device arrays (fpho_patch_replace_meta reads only the metadata
        fields; patch creation copies the device arrays)."""
        ptrs = {k: t.data_ptr() for k, t in (self.pixels or {}).items()
                if k not in self.__dict__}
        ptrs.update(pointers or {})
        return super().host_struct(residual=residual, pointers=ptrs)

    def _pixel_array(self, attr):
        a = self.__dict__.get(attr)
        if a is None and self.pixels is not None and attr in self.pixels:
            a = self.pixels[attr].cpu().numpy()
        return a if a is not None else getattr(self, attr)

    def split_pix(self, attr):
        """Per-exposure pieces of a pixel array (copied from the device when
        the patch holds it there)."""
        return np.split(self._pixel_array(attr), np.cumsum(self.exposure_N[:-1]))

    def split_band(self, attr):
        """Per-band pieces of a pixel array (copied from the device when the
        patch holds it there)."""
        return np.split(self._pixel_array(attr), np.cumsum(self.band_N_pix[:-1]))

    def pixels_to_host(self):
        """Copy the device pixel arrays into ``data``, ``ierr``, ``xpix``,
        ``ypix`` (numpy), as the host StorePatch holds them."""
        for k, t in self.pixels.items():
            setattr(self, k, t.cpu().numpy())
        return self

    def send_to_device(self):
        if self.pixels is None:
            raise RuntimeError("build_patch (or pack_pix) must run before send_to_device")
        ptrs = {k: t.data_ptr() for k, t in self.pixels.items()}
        self.device_patch = DevicePatch(self, return_residual=self.return_residual,
                                        device_pixels=ptrs)
        self._dirty_data = False
        return self.device_patch
