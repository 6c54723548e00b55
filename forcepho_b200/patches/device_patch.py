"""Device communication of patch data.

:class:`GPUPatchMixin` mirrors forcepho/patches/device_patch.py:260-393
(``send_to_device``, ``replace_device_meta_ptrs``,
``send_patchstruct_to_device``, ``swap_on_device``, ``retrieve_array``,
``free``, ``get_proposer`` and the ``device_patch`` attribute), backed by a
``fpho_patch`` handle of the C ABI instead of pycuda allocations.
:class:`DevicePatchMixin` adds the reference's fixed-source subtraction and
rendering helpers that are built on the same evaluation
(device_patch.py:113-254).
"""

import ctypes

import numpy as np

from .. import _lib
from ..proposal import GPUProposer

__all__ = ["DevicePatch", "DevicePatchMixin", "GPUPatchMixin"]

_ARRAY_CODE = {"data": 0, "residual": 1, "ierr": 2, "xpix": 3, "ypix": 4}


class DevicePatch:
    """Owner of one ``fpho_patch`` handle (device copy of a patch + workspace)."""

    def __init__(self, patch, return_residual=False, stream=None, device_pixels=None):
        """`device_pixels`: {"data", "ierr", "xpix", "ypix": device address}
        to create the patch from pixel arrays already on the device."""
        st = patch.host_struct(pointers=device_pixels)
        self._keep = st  # host arrays stay referenced by `patch`
        h = ctypes.c_void_p()
        create = "fpho_patch_create_device_pixels" if device_pixels else "fpho_patch_create"
        _lib.call(create, st.ctypes.data, int(patch.n_bands), int(bool(return_residual)), stream,
                  ctypes.byref(h))
        self.handle = h.value
        self.return_residual = bool(return_residual)

    def info(self):
        out = (ctypes.c_int64 * 7)()
        _lib.call("fpho_patch_info", self.handle, out)
        keys = ["n_bands", "n_exp", "npix", "n_sources", "n_radii", "n_tiles", "n_gauss"]
        return dict(zip(keys, list(out)))

    @property
    def device_struct(self):
        """Device address of the patch struct (device pointers inside)."""
        p = ctypes.c_void_p()
        _lib.call("fpho_patch_device_struct", self.handle, ctypes.byref(p))
        return p.value

    def set_config(self, variant, live_cap, stream=None):
        _lib.call("fpho_patch_set_config", self.handle, int(variant), int(live_cap), stream)

    def set_schedule(self, schedule):
        """0: one CTA per tile; 1: persistent CTAs, costliest tiles first."""
        _lib.call("fpho_patch_set_schedule", self.handle, int(schedule))

    def set_exact_residual(self, on=True, live_cap=160, stream=None):
        """Residual pass in the reference's float arithmetic (a parity
        diagnostic, see fpho_patch_set_exact_residual); switching it on
        selects the 64 x 4 tile variant that compiles it."""
        if on:
            self.set_config(3, live_cap, stream)
        _lib.call("fpho_patch_set_exact_residual", self.handle, int(bool(on)))

    def free(self):
        if getattr(self, "handle", None):
            _lib.lib.fpho_patch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class DevicePatchMixin:
    """Methods shared by device mixins (forcepho/patches/device_patch.py:23-257).

    ``subtract_fixed`` and ``design_matrix`` need the patch class to provide
    ``set_scene(catalog)`` and ``pack_meta(scene)`` (the reference's
    JadesPatch does; :class:`forcepho_b200.synth.SyntheticPatch` does for its
    own sources)."""

    def get_proposer(self):
        raise NotImplementedError

    def send_to_device(self):
        raise NotImplementedError

    def subtract_fixed(self, fixed, active=None, big=None, maxactive=15, swap_local=False,
                       big_scene_kwargs={}, **scene_kwargs):
        """Subtract fixed (and big) sources from the device data, block by block
        of at most `maxactive` sources, leaving the residual as the device data
        and the metadata of `active` (or of the last block) installed; returns
        (proposer, scene of the installed metadata).  As the reference's
        ``subtract_fixed`` (device_patch.py:113-191)."""
        scenes = []
        if big is not None:
            inds = np.arange(maxactive, len(big), maxactive)
            scenes.extend([self.set_scene(b, **big_scene_kwargs)
                           for b in np.array_split(np.asarray(big), inds)])
        if fixed is not None:
            inds = np.arange(maxactive, len(fixed), maxactive)
            scenes.extend([self.set_scene(b, **scene_kwargs)
                           for b in np.array_split(np.asarray(fixed), inds)])
        if active is not None:
            scenes.append(self.set_scene(active, **scene_kwargs))
        else:
            if not swap_local:
                raise ValueError("without `active` the installed metadata belong to a scene "
                                 "already subtracted; pass swap_local=True to accept that")
            scenes.append(scenes[-1])
        if not scenes:
            raise ValueError("No scenes to prepare!")
        proposer = self.get_proposer()
        self.return_residual = True
        self.pack_meta(scenes[0])
        self.free()
        self.send_to_device()  # the host pixel data, unsubtracted
        for i, scene in enumerate(scenes[1:]):
            proposer.evaluate_proposal(scenes[i].get_proposal(), patch=self)
            self.pack_meta(scene)
            self.swap_on_device()
        return proposer, scenes[-1]

    def design_matrix_device(self, proposal, stream=None):
        """Unit-flux model of every source of `proposal` (the scene whose
        metadata are installed) at every pixel: a float32 CUDA tensor
        (n_sources, npix) computed by ``fpho_patch_design_matrix``."""
        import torch
        prop = np.ascontiguousarray(proposal)
        ns = len(prop)
        dprop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
        X = torch.empty((ns, int(self.npix)), dtype=torch.float32, device="cuda")
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _lib.call("fpho_patch_design_matrix", self.device_patch.handle, dprop.data_ptr(), ns,
                  X.data_ptr(), s)
        return X

    def design_matrix(self, active=None, proposer=None, **scene_kwargs):
        """(Xes, ys): per band the design matrix X (n_source, n_pix_band) with
        Y[band] = f[band] . X[band] and the target data (the device data, e.g.
        after :meth:`subtract_fixed`), as the reference's ``design_matrix``
        (device_patch.py:193-238).  One launch builds every source's row."""
        scene = active if hasattr(active, "get_proposal") else \
            self.set_scene(active, **scene_kwargs)
        self.pack_meta(scene)
        self.replace_device_meta_ptrs()
        X = self.design_matrix_device(scene.get_proposal()).cpu().numpy()
        y = self.retrieve_array("data")
        cuts = np.cumsum(self.band_N_pix[:-1])
        return list(np.split(X, cuts, axis=1)), list(np.split(y, cuts))

    def render(self, proposal):
        """Model images (one flat array per exposure) of a proposal, as the
        reference's ``render`` (device_patch.py:240-254) but taking the
        packed proposal directly."""
        orig = self.return_residual
        if not orig or getattr(self, "device_patch", None) is None or \
                not self.device_patch.return_residual:
            self.return_residual = True
            self.free()
            self.send_to_device()
        proposer = self.get_proposer()
        chi2, derivs, residuals = proposer.evaluate_proposal(proposal, patch=self, unpack=True)
        data = self.split_pix("data")
        self.return_residual = orig
        return [d - r for d, r in zip(data, residuals)]


class GPUPatchMixin(DevicePatchMixin):
    """Mix-in for communicating patch data with the GPU through the C ABI."""

    def get_proposer(self):
        return GPUProposer()

    def send_to_device(self):
        """Copy every patch array to the device; returns ``self.device_patch``."""
        self.device_patch = DevicePatch(self, return_residual=self.return_residual)
        self._dirty_data = False
        return self.device_patch

    def replace_device_meta_ptrs(self):
        """Replace the device metadata with the currently packed host metadata."""
        st = self.host_struct()
        _lib.call("fpho_patch_replace_meta", self.device_patch.handle, st.ctypes.data, None)

    def send_patchstruct_to_device(self):
        """The device patch struct is refreshed by every C-ABI call that
        changes a pointer; this returns the handle for compatibility."""
        return self.device_patch

    def swap_on_device(self):
        """Install the packed metadata and make the device residual the data
        (device_patch.py:346-367)."""
        if not self.device_patch.return_residual:
            raise AssertionError("Must instantiate the Patch with `return_residual=True`")
        self.replace_device_meta_ptrs()
        _lib.call("fpho_patch_swap_data_residual", self.device_patch.handle, None)
        self._dirty_data = True
        return self.device_patch

    def retrieve_array(self, arrname="residual"):
        """Copy a pixel array (data, residual, ierr, xpix, ypix) to the host."""
        out = np.empty(self.npix, dtype=np.float32)
        _lib.call("fpho_patch_retrieve", self.device_patch.handle, _ARRAY_CODE[arrname],
                  out.ctypes.data, None)
        return out

    def free(self):
        dp = getattr(self, "device_patch", None)
        if dp is not None:
            dp.free()
        self.device_patch = None
