"""ctypes binding of ``libfpho.so`` (the C ABI declared in include/fpho.h).

The library is built in-tree by :mod:`forcepho_b200.build`.  It is loaded on
first use (the first access to ``lib`` or the first call through this
module), so that code which only needs the package's host-side pieces -- the
synthetic patches, the packing and the file readers -- does not map it.  If
it is missing it is compiled (nvcc is present wherever the package is built),
and if that is impossible the first use fails loudly: there is no CPU
fallback for the hot path.
"""

import ctypes
import os

import numpy as np

from . import build as _build

FPHO_OK = 0
FPHO_IO_HOST = 1
FPHO_WANT_RESIDUAL = 2
FPHO_CHI2_ONLY = 4

_ERRNAMES = {1: "INVALID", 2: "CUDA", 3: "NOMEM", 4: "LIMIT", 5: "STATE", 6: "KERNEL"}


class FphoError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code, func, msg):
        self.code = code
        super().__init__(f"{func} -> FPHO_ERR_{_ERRNAMES.get(code, code)}: {msg}")


def _load():
    path = _build.LIB
    if _build.needs_build():
        _build.build()
    if not os.path.exists(path):
        raise ImportError(f"forcepho_b200: CUDA library {path} is missing and could not be built")
    return ctypes.CDLL(path)

c_void_p = ctypes.c_void_p
c_int = ctypes.c_int
c_uint = ctypes.c_uint
c_int64_p = ctypes.POINTER(ctypes.c_int64)

_SIGS = {
    "fpho_last_error": (ctypes.c_char_p, []),
    "fpho_abi_version": (c_int, []),
    "fpho_sizeof": (c_int, [c_int]),
    "fpho_patch_create": (c_int, [c_void_p, c_int, c_int, c_void_p, ctypes.POINTER(c_void_p)]),
    "fpho_patch_replace_meta": (c_int, [c_void_p, c_void_p, c_void_p]),
    "fpho_patch_swap_data_residual": (c_int, [c_void_p, c_void_p]),
    "fpho_patch_retrieve": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "fpho_patch_device_struct": (c_int, [c_void_p, ctypes.POINTER(c_void_p)]),
    "fpho_patch_info": (c_int, [c_void_p, c_int64_p]),
    "fpho_patch_free": (c_int, [c_void_p]),
    "fpho_patch_create_device_pixels": (c_int, [c_void_p, c_int, c_int, c_void_p,
                                                ctypes.POINTER(c_void_p)]),
    "fpho_store_create": (c_int, [c_int, c_int, c_int, c_int, ctypes.POINTER(c_void_p)]),
    "fpho_store_add_exposure": (c_int, [c_void_p, c_void_p, c_int, c_void_p,
                                        ctypes.POINTER(c_int)]),
    "fpho_store_info": (c_int, [c_void_p, c_int64_p]),
    "fpho_store_count": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "fpho_store_gather": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, ctypes.c_float,
                                  c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int64,
                                  c_void_p, c_void_p, c_void_p]),
    "fpho_store_free": (c_int, [c_void_p]),
    "fpho_store_time_gather": (c_int, [c_void_p, c_int]),
    "fpho_store_last_gather_ms": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "fpho_patch_set_config": (c_int, [c_void_p, c_int, c_int, c_void_p]),
    "fpho_patch_set_schedule": (c_int, [c_void_p, c_int]),
    "fpho_patch_set_exact_residual": (c_int, [c_void_p, c_int]),
    "fpho_patch_set_test_stall": (c_int, [c_void_p, c_int]),
    "fpho_patch_design_matrix": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "fpho_patch_flux_normal_equations": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                                 c_void_p]),
    "fpho_patch_optimize_fluxes": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                           c_void_p, c_void_p]),
    "fpho_variant_info": (c_int, [c_int, ctypes.POINTER(c_int)]),
    "fpho_variant_shape": (c_int, [c_int, ctypes.POINTER(c_int)]),
    "fpho_patch_count_pairs": (c_int, [c_void_p, c_int, ctypes.POINTER(ctypes.c_longlong)]),
    "fpho_patch_error_word": (c_int, [c_void_p, ctypes.POINTER(c_int)]),
    "fpho_evaluate_proposal": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                       c_uint, c_void_p]),
    "fpho_EvaluateProposal": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                      c_void_p]),
    "fpho_evaluate_proposal_noalloc": (c_int, [c_void_p, c_int, c_int, ctypes.c_int64, c_int,
                                               c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                                               c_void_p]),
    "fpho_batch_create": (c_int, [c_void_p, c_int, c_int, c_void_p, ctypes.POINTER(c_void_p)]),
    "fpho_batch_info": (c_int, [c_void_p, c_int64_p]),
    "fpho_batch_create_config": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p,
                                         ctypes.POINTER(c_void_p)]),
    "fpho_batch_variants": (c_int, [ctypes.POINTER(c_int), c_int]),
    "fpho_batch_config": (c_int, [c_void_p, ctypes.POINTER(c_int)]),
    "fpho_batch_evaluate": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_uint, c_void_p]),
    "fpho_batch_count_pairs": (c_int, [c_void_p, c_int, ctypes.POINTER(ctypes.c_longlong)]),
    "fpho_batch_time_tiles": (c_int, [c_void_p, c_int]),
    "fpho_batch_last_tile_ms": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "fpho_batch_error_word": (c_int, [c_void_p, ctypes.POINTER(c_int)]),
    "fpho_batch_free": (c_int, [c_void_p]),
    "fpho_spline_create": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p,
                                   ctypes.c_double, c_void_p, ctypes.POINTER(c_void_p)]),
    "fpho_spline_free": (c_int, [c_void_p]),
    "fpho_build_proposal": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "fpho_build_proposal_batch": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                          c_void_p, c_void_p]),
    "fpho_spline_points": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "fpho_build_proposal_bounded": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                            c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "fpho_bounded_lnp_grad": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                      c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                      c_int, c_void_p, c_void_p]),
    "fpho_patch_time_tiles": (c_int, [c_void_p, c_int]),
    "fpho_patch_image_gaussians": (c_int, [c_void_p, c_int, c_void_p, c_int,
                                           ctypes.POINTER(c_int)]),
    "fpho_patch_last_tile_ms": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "fpho_probe_launch": (c_int, [c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
}


def _bind(L):
    missing = []
    for name, (res, args) in _SIGS.items():
        try:
            f = getattr(L, name)
        except AttributeError:
            missing.append(name)
            continue
        f.restype = res
        f.argtypes = args
    if missing:
        raise ImportError(f"libfpho.so lacks symbols: {missing}")


_loaded = None


def get():
    """The loaded and bound library (loads it on the first call)."""
    global _loaded
    if _loaded is None:
        L = _load()
        _bind(L)
        _loaded = L
        globals()["lib"] = L
    return _loaded


def __getattr__(name):
    if name == "lib":
        return get()
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def last_error():
    return get().fpho_last_error().decode(errors="replace")


def check(rc, func="fpho"):
    if rc != FPHO_OK:
        raise FphoError(rc, func, last_error())
    return rc


def call(name, *args):
    """Call a C-ABI function and raise FphoError on a non-zero status."""
    return check(getattr(get(), name)(*args), name)


def variants():
    """List of (threads per CTA, pixels per thread) of the compiled tile kernels."""
    out = (c_int * 2)()
    L = get()
    n = L.fpho_variant_info(0, out)
    res = []
    for v in range(n):
        L.fpho_variant_info(v, out)
        res.append((out[0], out[1]))
    return res


def variant_shapes():
    """List of (threads per CTA, pixels per tile, warps sharing a tile's
    Gaussians -- 0 for the classic body) of the compiled tile kernels."""
    out = (c_int * 3)()
    L = get()
    n = L.fpho_variant_shape(0, out)
    res = []
    for v in range(n):
        L.fpho_variant_shape(v, out)
        res.append((out[0], out[1], out[2]))
    return res


def ptr(a):
    """Address of a numpy array or torch tensor (or an int)."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
