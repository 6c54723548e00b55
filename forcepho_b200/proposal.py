"""Host interface to evaluate a proposal on the GPU.

Mirrors forcepho/proposal.py: ``ProposerBase``, ``GPUProposer`` (alias
``Proposer``) and the ``source_struct_dtype`` / ``response_struct_dtype``
numpy layouts of the device ABI (forcepho/proposal.py:229-244,
forcepho/src/proposal.cu:13-39).  ``GPUProposer.evaluate_proposal`` keeps the
reference's signature and return values (forcepho/proposal.py:96-152) and
calls ``fpho_evaluate_proposal`` of the C ABI instead of launching a pycuda
kernel.
"""

import sys

import numpy as np

from . import _lib
from .kernel_limits import MAXBANDS, MAXRADII, MAXSOURCES, NPARAMS

__all__ = ["ProposerBase", "Proposer", "GPUProposer",
           "source_struct_dtype", "response_struct_dtype"]

source_float_dt = np.float32
source_struct_dtype = np.dtype([('ra', source_float_dt),
                                ('dec', source_float_dt),
                                ('q', source_float_dt),
                                ('pa', source_float_dt),
                                ('nsersic', source_float_dt),
                                ('rh', source_float_dt),
                                ('fluxes', source_float_dt, MAXBANDS),
                                ('mixture_amplitudes', source_float_dt, MAXRADII),
                                ('damplitude_drh', source_float_dt, MAXRADII),
                                ('damplitude_dnsersic', source_float_dt, MAXRADII)],
                               align=True)

response_float_dt = source_float_dt
response_struct_dtype = np.dtype([('dchi2_dparam', response_float_dt,
                                   NPARAMS * MAXSOURCES)], align=True)


class ProposerBase:

    def __init__(self):
        pass

    def evaluate_proposal(self, proposal, **kwargs):
        raise NotImplementedError

    def unpack_residuals(self, residuals_flat, patch, reshape=False):
        """Split flat, padded residuals into one array per exposure (and, with
        ``reshape``, drop padding and reshape to the original stamp shapes),
        as forcepho/proposal.py:38-52."""
        residuals = np.split(residuals_flat, np.cumsum(patch.exposure_N)[:-1])
        if reshape:
            for e, residual in enumerate(residuals):
                residual = residual[:patch.original_sizes[e]]
                residuals[e] = residual.reshape(patch.original_shapes[e])
        return residuals


class GPUProposer(ProposerBase):
    """Evaluate proposals with the forcepho_b200 CUDA kernels.

    The constructor accepts the reference's arguments.  ``thread_block``,
    ``shared_size``, ``max_registers``, ``show_ptxas``, ``debug``,
    ``kernel_name`` and ``kernel_fn`` configured the reference's runtime
    compilation of its .cu file; here the kernels are compiled ahead of time
    and their launch shape is chosen per patch (see
    :mod:`forcepho_b200.autotune`), so those arguments are accepted and
    ignored.  ``chi_dtype`` must be float64 (the chi2 accumulator type).
    """

    def __init__(self, patch=None, thread_block=1024, shared_size=48000,
                 max_registers=64, show_ptxas=False, debug=False,
                 kernel_name='EvaluateProposal', chi_dtype=np.float64,
                 kernel_fn='compute_gaussians_kernel.cu'):
        if np.dtype(chi_dtype) != np.float64:
            raise ValueError("chi_dtype must be float64")
        self.block = (thread_block, 1, 1)
        self.shared_size = shared_size
        self.chi_dtype = np.float64
        self.patch = patch

    def evaluate_proposal(self, proposal, patch=None, verbose=False, unpack=True):
        """Evaluate the likelihood of a parameter proposal.

        Parameters
        ----------
        proposal : ndarray of dtype ``source_struct_dtype``, shape (n_sources,)

        Returns
        -------
        chi2 : ndarray of shape (n_bands,), float64
            Per-band sum of (r*ie - d*ie)(r*ie + d*ie), r = data - model.
        chi2_derivs : ndarray of shape (n_bands, n_sources, 7), float32
            d chi2 / d (flux, ra, dec, q, pa, sersic, rh) per band and source.
        residuals : list of ndarray
            Per-exposure residual (data - model); only if
            ``patch.return_residual``.
        """
        if patch is None:
            patch = self.patch
        dev = patch.device_patch
        n_bands, n_sources = patch.n_bands, patch.n_sources
        proposal = np.ascontiguousarray(proposal, dtype=source_struct_dtype)
        if proposal.shape[0] != n_sources:
            raise ValueError(f"proposal has {proposal.shape[0]} sources, patch has {n_sources}")
        chi_out = np.empty(n_bands, dtype=np.float64)
        derivs = np.empty((n_bands, n_sources, NPARAMS), dtype=np.float32)
        flags = _lib.FPHO_IO_HOST
        if patch.return_residual:
            flags |= _lib.FPHO_WANT_RESIDUAL
        if verbose:
            print(f"evaluate_proposal: {n_bands} bands, {n_sources} sources, "
                  f"{patch.npix} pixels", file=sys.stderr, flush=True)
        _lib.call("fpho_evaluate_proposal", dev.handle, proposal.ctypes.data, n_sources,
                  chi_out.ctypes.data, derivs.ctypes.data, NPARAMS * n_sources, flags, None)
        if patch.return_residual:
            residuals = patch.retrieve_array("residual")
            if unpack:
                residuals = self.unpack_residuals(residuals, patch)
            return chi_out, derivs, residuals
        return chi_out, derivs


class Proposer(GPUProposer):
    """Alias kept for compatibility with the reference."""
    pass
