"""Patch packing and device communication (mirrors forcepho.patches)."""

from .patch import PatchBase, PSF_COLS, PSF_DTYPE  # noqa: F401
from .device_patch import DevicePatch, DevicePatchMixin, GPUPatchMixin  # noqa: F401
