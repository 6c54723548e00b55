"""Host-side patch data model.

:class:`PatchBase` mirrors the reference's ``PatchBase``
(forcepho/patches/patch.py:20-197): the numpy arrays a patch is packed into and
the ``patch_struct_dtype`` of pointers and counts, which is byte-compatible
with the ``Patch`` struct of the device ABI (forcepho/src/patch.cc:23-99,
``fpho_patch_struct`` in include/fpho.h).
"""

import numpy as np

__all__ = ["PatchBase", "Patch", "PSF_COLS", "PSF_DTYPE"]

# PSF Gaussian columns, as forcepho/patches/storage.py:35-36
PSF_COLS = ["amp", "xcen", "ycen", "Cxx", "Cyy", "Cxy"]
PSF_DTYPE = np.dtype([(c, np.float32) for c in PSF_COLS] + [("sersic_bin", np.int32)])


class PatchBase:
    """Arrays of one patch packed for the device.

    Parameters
    ----------
    return_residual : bool
        Whether evaluations also write the residual image (data - model).
    pix_dtype, meta_dtype : numpy dtype
        Must be float32 (the device ABI is single precision).
    """

    ptr_dtype = np.uintp
    pdt = np.dtype([('data', ptr_dtype),
                    ('ierr', ptr_dtype),
                    ('xpix', ptr_dtype),
                    ('ypix', ptr_dtype),
                    ('residual', ptr_dtype),
                    ('exposure_start', ptr_dtype),
                    ('exposure_N', ptr_dtype),
                    ('band_start', ptr_dtype),
                    ('band_N', ptr_dtype),
                    ('n_sources', np.int32),
                    ('n_radii', np.int32),
                    ('rad2', ptr_dtype),
                    ('D', ptr_dtype),
                    ('crpix', ptr_dtype),
                    ('crval', ptr_dtype),
                    ('CW', ptr_dtype),
                    ('G', ptr_dtype),
                    ('n_psf_per_source', ptr_dtype),
                    ('psfgauss', ptr_dtype),
                    ('psfgauss_start', ptr_dtype)],
                   align=True)
    patch_struct_dtype = pdt
    meta_names = ["n_sources", "n_radii", "rad2",
                  "D", "crpix", "crval", "CW", "G",
                  "n_psf_per_source", "psfgauss", "psfgauss_start"]

    # dtype of every array field, used to coerce before taking pointers
    array_dtypes = dict(data=np.float32, ierr=np.float32, xpix=np.float32, ypix=np.float32,
                        residual=np.float32, exposure_start=np.int32, exposure_N=np.int32,
                        band_start=np.int16, band_N=np.int16, rad2=np.float32, D=np.float32,
                        crpix=np.float32, crval=np.float32, CW=np.float32, G=np.float32,
                        n_psf_per_source=np.int32, psfgauss=PSF_DTYPE, psfgauss_start=np.int32)

    def __init__(self, return_residual=False, pix_dtype=np.float32, meta_dtype=np.float32):
        if np.dtype(pix_dtype) != np.float32 or np.dtype(meta_dtype) != np.float32:
            raise ValueError("the device ABI is float32: pix_dtype and meta_dtype must be float32")
        self.pix_dtype = np.float32
        self.meta_dtype = np.float32
        self.return_residual = return_residual
        self._dirty_data = True

    @property
    def npix(self):
        try:
            return self.xpix.shape[0]
        except AttributeError:
            return 0

    @property
    def n_bands(self):
        return len(self.band_start)

    @property
    def n_exp(self):
        return len(self.exposure_start)

    @property
    def size(self):
        s = 0
        for arrname in self.patch_struct_dtype.names:
            a = getattr(self, arrname, None)
            if isinstance(a, np.ndarray):
                s += a.nbytes
        return s

    @property
    def band_N_pix(self):
        """Pixels (with padding) of each band."""
        out = np.zeros(self.n_bands, dtype=np.int64)
        for b in range(self.n_bands):
            e0, n = int(self.band_start[b]), int(self.band_N[b])
            out[b] = int(np.sum(self.exposure_N[e0:e0 + n]))
        return out

    def clear(self):
        for arrname in self.patch_struct_dtype.names:
            try:
                delattr(self, arrname)
            except AttributeError:
                pass

    def free(self):
        pass

    def build_patch(self, npix=1, n_sources=1, n_radii=1, n_bands=1, n_exp=1):
        """Allocate every array with the proper shape and dtype (as the
        reference's ``build_patch``, forcepho/patches/patch.py:121-197)."""
        self.xpix = np.zeros(npix, dtype=np.float32)
        self.ypix = np.zeros(npix, dtype=np.float32)
        self.data = np.zeros(npix, dtype=np.float32)
        self.ierr = np.zeros(npix, dtype=np.float32)
        self.band_start = np.zeros(n_bands, dtype=np.int16)
        self.band_N = np.zeros(n_bands, dtype=np.int16)
        self.exposure_start = np.zeros(n_exp, dtype=np.int32)
        self.exposure_N = np.zeros(n_exp, dtype=np.int32)
        self.n_sources = n_sources
        self.n_radii = n_radii
        self.rad2 = np.zeros(n_radii, dtype=np.float32)
        self.D = np.zeros((n_exp, n_sources, 2, 2), dtype=np.float32)
        self.CW = np.zeros((n_exp, n_sources, 2, 2), dtype=np.float32)
        self.crpix = np.zeros((n_exp, n_sources, 2), dtype=np.float32)
        self.crval = np.zeros((n_exp, n_sources, 2), dtype=np.float32)
        self.G = np.zeros(n_exp, dtype=np.float32)
        self.n_psf_per_source = np.zeros(n_bands, dtype=np.int32)
        self.psfgauss = np.zeros(0, dtype=PSF_DTYPE)
        self.psfgauss_start = np.zeros(n_exp, dtype=np.int32)

    def coerce_arrays(self):
        """Make every array C-contiguous with the ABI dtype (in place)."""
        for name, dt in self.array_dtypes.items():
            a = getattr(self, name, None)
            if a is None:
                continue
            setattr(self, name, np.ascontiguousarray(a, dtype=dt))

    def host_struct(self, residual=None, pointers=None):
        """A ``patch_struct_dtype`` record holding HOST pointers to this
        patch's arrays (the form :func:`fpho_patch_create` reads).
        `pointers` ({field: address}) overrides fields, e.g. device pixel
        arrays for ``fpho_patch_create_device_pixels``."""
        self.coerce_arrays()
        pointers = pointers or {}
        st = np.zeros(1, dtype=self.patch_struct_dtype)
        for name in self.patch_struct_dtype.names:
            if name in pointers:
                st[name] = pointers[name]
            elif self.patch_struct_dtype[name] == self.ptr_dtype:
                if name == "residual":
                    st[name] = 0 if residual is None else residual.ctypes.data
                else:
                    st[name] = getattr(self, name).ctypes.data
            else:
                st[name] = getattr(self, name)
        return st

    def split_pix(self, attr):
        """Split a pixel array into one array per exposure."""
        arr = getattr(self, attr)
        return np.split(arr, np.cumsum(self.exposure_N[:-1]))

    def split_band(self, attr):
        """Split a pixel array into one array per band."""
        arr = getattr(self, attr)
        return np.split(arr, np.cumsum(self.band_N_pix[:-1]))


class Patch(PatchBase):
    """A patch whose per-scene metadata is packed from exposure WCSs, a PSF
    store and a Sersic spline table (forcepho/patches/patch.py:200-424:
    ``pack_meta``, ``_pack_source_metadata``, ``_pack_astrometry``,
    ``_pack_fluxcal``, ``_pack_psf``, ``set_scene``, ``zerocoords``).

    Subclasses fill the pixel arrays and the exposure lists ``wcses``,
    ``hdrs``, ``bands``, ``bandlist``, ``n_exp_per_band``.

    Parameters
    ----------
    psfstore : path of a PSF store (HDF5), or ""
    splinedata : path of a Sersic spline table (forcepho's ``.h5`` or this
        package's ``.npz``); "" uses the packaged table
    spline_smoothing : smoothing of the amplitude splines
    """

    def __init__(self, psfstore="", splinedata="", spline_smoothing=None,
                 return_residual=False, meta_dtype=np.float32, pix_dtype=np.float32, debug=0):
        super().__init__(return_residual=return_residual, meta_dtype=meta_dtype,
                         pix_dtype=pix_dtype)
        from .storage import PSFStore
        self.debug = debug
        self.psfstore = PSFStore(psfstore) if psfstore else None
        self.splinedata = splinedata
        self.spline_smoothing = spline_smoothing
        self.patch_reference_coordinates = np.zeros(2)
        self._table = None

    @property
    def table(self):
        from ..sources import SersicTable, default_table
        if self._table is None:
            self._table = (SersicTable.from_file(self.splinedata, self.spline_smoothing)
                           if self.splinedata else default_table())
        return self._table

    def set_scene(self, sourcecat, splinedata=None):
        """A Scene of the catalog rows: fluxes from the columns named by
        ``bandlist``, then ra, dec, q, pa, sersic, rhalf."""
        from ..sources import SHAPE_COLS, Scene, SersicTable
        table = SersicTable.from_file(splinedata, self.spline_smoothing) if splinedata \
            else self.table
        cat = np.atleast_1d(sourcecat)
        cols = list(self.bandlist) + SHAPE_COLS
        params = np.stack([np.asarray(cat[c], dtype=np.float64) for c in cols], axis=-1)
        return Scene(len(cat), len(self.bandlist), table, params=params)

    def zerocoords(self, scene, sky_zero=None):
        """Subtract the (median, by default) source position from the
        scene's positions in place and return it (patch.py:425-456)."""
        nb = scene.n_bands
        if sky_zero is None:
            sky_zero = np.array([np.median(scene.params[:, nb]),
                                 np.median(scene.params[:, nb + 1])])
        zero = np.array(sky_zero, dtype=np.float64)
        self.patch_reference_coordinates = zero
        scene.params[:, nb] -= zero[0]
        scene.params[:, nb + 1] -= zero[1]
        return zero

    def unzerocoords(self, scene):
        nb = scene.n_bands
        zero = self.patch_reference_coordinates
        scene.params[:, nb] += zero[0]
        scene.params[:, nb + 1] += zero[1]
        return scene

    def pack_meta(self, scene):
        self.patch_reference_coordinates = self.zerocoords(scene)
        self.n_sources = len(scene)
        self._pack_source_metadata(scene)
        self._pack_astrometry(self.wcses, scene)
        self._pack_fluxcal(self.hdrs)
        self._pack_psf(self.bands, self.wcses, scene)
        self.scene = scene

    def _pack_source_metadata(self, scene, dtype=None):
        self.n_sources = len(scene)
        self.n_radii = scene.table.n_radii
        self.rad2 = (scene.table.radii ** 2).astype(np.float32)

    def _pack_astrometry(self, wcses, scene, dtype=None):
        from ..wcs import scale_at_sky
        ns, nb = len(scene), scene.n_bands
        self.D = np.empty((self.n_exp, ns, 2, 2), dtype=np.float32)
        self.CW = np.empty((self.n_exp, ns, 2, 2), dtype=np.float32)
        self.crpix = np.empty((self.n_exp, ns, 2), dtype=np.float32)
        self.crval = np.empty((self.n_exp, ns, 2), dtype=np.float32)
        ra0, dec0 = self.patch_reference_coordinates
        sky = np.stack([scene.params[:, nb] + ra0, scene.params[:, nb + 1] + dec0], axis=-1)
        # cos(dec) of each source, as scale_at_sky computes it (scalar calls)
        cosd = np.array([np.cos(np.deg2rad(d)) for d in sky[:, 1]])
        for j, wcs in enumerate(wcses):
            if getattr(wcs, "has_distortion", True):
                for i in range(ns):
                    CW_mat, D_mat = scale_at_sky(sky[i], wcs)
                    self.D[j, i] = D_mat
                    self.CW[j, i] = CW_mat
            else:
                # scale_at_sky's linear branch for every source at once: D is
                # the same for all sources, CW = (3600 D) diag(cos dec, 1), whose
                # matrix product has exact zero and unit terms, so the columns
                # are scaled elementwise with the same results
                D_mat = getattr(wcs, "_linear_D", None)     # the same for every scene
                if D_mat is None:
                    D_mat = np.linalg.inv(wcs.pixel_scale_matrix * 3600.0)
                    try:
                        wcs._linear_D = D_mat
                    except AttributeError:
                        pass
                A = D_mat * 3600.0
                self.D[j] = D_mat
                self.CW[j, :, :, 0] = A[None, :, 0] * cosd[:, None]
                self.CW[j, :, :, 1] = A[None, :, 1]
            self.crval[j] = sky - self.patch_reference_coordinates
        # source positions in every exposure's pixels: one pass over a stack of
        # TAN WCSs (elementwise the same arithmetic as one call per exposure)
        from ..wcs import TanWCS, TanWCSStack
        if wcses and all(isinstance(w, TanWCS) for w in wcses):
            x, y = TanWCSStack(wcses).world_to_pixel_values(sky[:, 0], sky[:, 1])
            self.crpix[:] = np.stack([x, y], axis=-1)
        else:
            for j, wcs in enumerate(wcses):
                x, y = wcs.world_to_pixel_values(sky[:, 0], sky[:, 1])
                self.crpix[j] = np.stack([x, y], axis=-1)

    def _pack_fluxcal(self, hdrs, tweakphot=None, dtype=None):
        self.G = np.ones(self.n_exp, dtype=np.float32)
        if tweakphot:
            for j, hdr in enumerate(hdrs):
                self.G[j] = hdr[tweakphot]

    def _pack_psf(self, bands, wcses, scene, dtype=None, psf_dtype=None):
        ns = len(scene)
        npsf = [self.psfstore.n_psf_per_source(b) for b in self.bandlist]
        self.n_psf_per_source = np.array(npsf, dtype=np.int32)
        self.psfgauss_start = np.zeros(self.n_exp, dtype=np.int32)
        n_psfgauss = int((self.n_psf_per_source * np.asarray(self.n_exp_per_band) * ns).sum())
        self.psfgauss = np.empty(n_psfgauss, dtype=PSF_DTYPE)
        blocks, tiled, s = [], {}, 0
        for e in range(self.n_exp):      # every source of an exposure gets its band's rows
            if bands[e] not in tiled:
                tiled[bands[e]] = np.tile(self.psfstore.lookup(bands[e]), ns)
            self.psfgauss_start[e] = s
            blocks.append(tiled[bands[e]])
            s += len(tiled[bands[e]])
        assert s == n_psfgauss
        self.psfgauss = np.concatenate(blocks).astype(PSF_DTYPE, copy=False) if blocks \
            else self.psfgauss
