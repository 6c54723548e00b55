"""The reference's own CUDA kernel, launched on the device copy of a patch.
TEST INFRASTRUCTURE ONLY (tests/; the GPU baseline of the benchmark figures).

oracle/Makefile compiles forcepho/src/compute_gaussians_kernel.cu, unchanged
and with the reference's nvcc options, together with oracle/refgpu_launch.cu
into oracle/_ref/librefgpu.so.  :func:`evaluate` launches it as
GPUProposer.evaluate_proposal does (forcepho/proposal.py:96-152): grid =
n_bands, 1024 threads, dynamic shared memory sized for the band with the most
image Gaussians; outputs chi2[n_bands] (double) and Response[n_bands]
(float dchi2_dparam[MAXSOURCES * 7]).
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "librefgpu.so")
_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.refgpu_launch.argtypes = [vp, vp, vp, vp, ip, ip, ip, ip, vp]
        L.refgpu_launch.restype = ip
        L.refgpu_shared_bytes.argtypes = [ip]
        L.refgpu_shared_bytes.restype = ip
        L.refgpu_max_sources.restype = ip
        _lib = L
    return _lib


def max_sources():
    return lib().refgpu_max_sources()


def evaluate(dev_struct, dev_proposal, dev_chi2, dev_response, n_bands, n_sources,
             max_gauss_band, stream=None, threads=1024):
    """Enqueue the reference kernel on device pointers (no synchronization)."""
    rc = lib().refgpu_launch(dev_struct, dev_proposal, dev_chi2, dev_response, int(n_bands),
                             int(n_sources), int(max_gauss_band), int(threads), stream)
    if rc != 0:
        raise RuntimeError(f"reference kernel launch refused or failed (code {rc})")


def max_gauss_band(patch):
    """Most image Gaussians (n_sources * n_psf_per_source) of any band."""
    return int(patch.n_sources) * int(np.max(patch.n_psf_per_source))
