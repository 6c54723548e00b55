"""Proposals built on the device.

:class:`DeviceSersicTable` uploads the bicubic B-splines of a
:class:`forcepho_b200.sources.SersicTable` (scipy's knots and coefficients)
and builds ``fpho_source`` proposals from a device parameter tensor in the
reference's Scene order (``Scene.get_proposal`` / ``Galaxy.proposal``,
forcepho/sources.py:80-97, 607-694), so that a sampler step never returns to
the host.
"""

import ctypes

import numpy as np
import torch

from . import _lib
from .proposal import source_struct_dtype
from .sources import default_table

__all__ = ["DeviceSersicTable", "SOURCE_BYTES"]

SOURCE_BYTES = source_struct_dtype.itemsize


def _stream():
    return torch.cuda.current_stream().cuda_stream


class DeviceSersicTable:
    """The Sersic amplitude splines of ``table`` on the current CUDA device."""

    def __init__(self, table=None):
        self.table = table or default_table()
        tx, ty, c = self.table.knots_and_coeffs()
        self._tx = np.ascontiguousarray(tx, dtype=np.float64)
        self._ty = np.ascontiguousarray(ty, dtype=np.float64)
        self._c = np.ascontiguousarray(c, dtype=np.float64)
        self._r = np.ascontiguousarray(self.table.radii, dtype=np.float64)
        h = ctypes.c_void_p()
        _lib.call("fpho_spline_create", self._tx.ctypes.data, len(self._tx),
                  self._ty.ctypes.data, len(self._ty), self._c.ctypes.data, len(self._r),
                  self._r.ctypes.data, float(self.table.sersic_range[0]), _stream(),
                  ctypes.byref(h))
        self.handle = h.value
        self.n_radii = len(self._r)

    def empty_proposal(self, n_sources):
        """A device byte buffer holding ``n_sources`` fpho_source records."""
        return torch.zeros(n_sources * SOURCE_BYTES, dtype=torch.uint8, device="cuda")

    def build_proposal(self, theta, n_bands, out=None):
        """theta: float64 CUDA tensor (n_sources, n_bands + 6), Scene order.
        Returns (or fills) the device proposal byte buffer."""
        if theta.dtype != torch.float64 or not theta.is_cuda:
            raise TypeError("theta must be a float64 CUDA tensor")
        theta = theta.contiguous()
        n_sources = theta.numel() // (n_bands + 6)
        if n_sources * (n_bands + 6) != theta.numel():
            raise ValueError("theta size is not a multiple of n_bands + 6")
        if out is None:
            out = self.empty_proposal(n_sources)
        _lib.call("fpho_build_proposal", self.handle, theta.data_ptr(), n_sources, n_bands,
                  out.data_ptr(), _stream())
        return out

    def build_proposal_batch(self, theta, src_bands, src_offset, out):
        """Proposals of many patches: source s has ``src_bands[s]`` bands and
        parameters at ``theta[src_offset[s]:]`` (int32 / int64 CUDA tensors)."""
        n = src_bands.numel()
        _lib.call("fpho_build_proposal_batch", self.handle, theta.data_ptr(), n,
                  src_bands.data_ptr(), src_offset.data_ptr(), out.data_ptr(), _stream())
        return out

    def points(self, x, y):
        """Spline values and (d/dsersic, d/drh) at points: (m, n_radii, 3) float64."""
        x = torch.as_tensor(x, dtype=torch.float64, device="cuda").contiguous()
        y = torch.as_tensor(y, dtype=torch.float64, device="cuda").contiguous()
        out = torch.empty((x.numel(), self.n_radii, 3), dtype=torch.float64, device="cuda")
        _lib.call("fpho_spline_points", self.handle, x.data_ptr(), y.data_ptr(), x.numel(),
                  out.data_ptr(), _stream())
        return out

    def free(self):
        if getattr(self, "handle", None):
            _lib.lib.fpho_spline_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def proposal_bytes_to_struct(buf):
    """Host copy of a device proposal buffer as a ``source_struct_dtype`` array."""
    return buf.cpu().numpy().view(source_struct_dtype).copy()
