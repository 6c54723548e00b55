"""The C-ABI library loads and exports every entry point include/fpho.h
declares; struct layouts agree with the numpy dtypes; host-side validation
rejects bad descriptors with status codes (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden

HEADER = os.path.join(ROOT, "include", "fpho.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"FPHO_API\s+[\w\s\*]*?\b(fpho_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "fpho_evaluate_proposal" in syms and "fpho_patch_create" in syms
    assert len(syms) >= 15


def test_library_exports_every_declared_symbol():
    from forcepho_b200 import _lib
    for s in declared_symbols():
        assert hasattr(_lib.lib, s), s


def test_struct_sizes_match_numpy_layouts():
    from forcepho_b200 import _lib
    from forcepho_b200.patches.patch import PatchBase, PSF_DTYPE
    from forcepho_b200.proposal import source_struct_dtype, response_struct_dtype
    assert _lib.lib.fpho_sizeof(0) == PatchBase.patch_struct_dtype.itemsize == 152
    assert _lib.lib.fpho_sizeof(1) == source_struct_dtype.itemsize == 264
    assert _lib.lib.fpho_sizeof(2) == PSF_DTYPE.itemsize == 28
    assert _lib.lib.fpho_sizeof(3) == response_struct_dtype.itemsize == 840


def test_oracle_struct_sizes():
    from oracle import oracle as O
    L = O.lib()
    assert L.fpo_sizeof_patch() == 152 and L.fpo_sizeof_source() == 264
    assert L.fpo_sizeof_psfgauss() == 28


def _create(st, n_bands):
    from forcepho_b200 import _lib
    h = ctypes.c_void_p()
    rc = _lib.lib.fpho_patch_create(st.ctypes.data if st is not None else None, n_bands, 0, None,
                                    ctypes.byref(h))
    return rc, _lib.last_error(), h


def test_create_rejects_null_and_bad_band_count():
    rc, msg, h = _create(None, 1)
    assert rc == 1 and "NULL" in msg and not h.value
    P, prop, d = load_golden("single_seed1")
    rc, msg, h = _create(P.host_struct(), 0)
    assert rc == 4 and "n_bands" in msg
    rc, msg, h = _create(P.host_struct(), 31)
    assert rc == 4


def test_create_rejects_negative_counts():
    P, prop, d = load_golden("mini_3src_2band")
    P.band_N = P.band_N.copy()
    P.band_N[1] = -1
    rc, msg, h = _create(P.host_struct(), 2)
    assert rc == 1 and "negative" in msg


def test_create_rejects_overlapping_bands():
    P, prop, d = load_golden("mini_3src_2band")
    P.band_start = np.array([0, 1], dtype=np.int16)
    rc, msg, h = _create(P.host_struct(), 2)
    assert rc == 1 and "belongs to bands" in msg


def test_create_rejects_bad_radius_bin():
    P, prop, d = load_golden("single_seed1")
    P.psfgauss = P.psfgauss.copy()
    P.psfgauss["sersic_bin"][3] = 99
    rc, msg, h = _create(P.host_struct(), 1)
    assert rc in (1, 2)   # 2 only if the pixel upload already needed a GPU


def test_variants_listed():
    """Classic shapes: whole warps, an even number of pixels per thread.
    Gaussian-split shapes: NW warps that each hold the whole tile, an even
    number of pixels per thread (32 K pixels per tile)."""
    from forcepho_b200 import _lib
    v = _lib.variants()
    shapes = _lib.variant_shapes()
    assert len(v) == 14 and len(shapes) == len(v)
    for (nt, k), (nt2, tile, split) in zip(v, shapes):
        assert nt == nt2 and nt % 32 == 0 and k == tile // nt
        if split == 0:
            assert k % 2 == 0 and tile == nt * k
        else:
            assert nt == 32 * split and tile % 64 == 0
    assert any(s > 0 for _, _, s in shapes)


def test_store_and_device_pixel_create_reject_bad_arguments():
    """Host-side checks of the exposure store and of
    fpho_patch_create_device_pixels, made before any CUDA call."""
    from forcepho_b200 import _lib
    L = _lib.lib
    h = ctypes.c_void_p()
    assert L.fpho_store_create(100, 64, 8, 1, ctypes.byref(h)) == 1 and not h.value  # 100 % 8
    assert "multiples" in _lib.last_error()
    assert L.fpho_store_create(64, 64, 0, 1, ctypes.byref(h)) == 1
    assert L.fpho_store_create(40000, 40000, 8, 1, ctypes.byref(h)) == 4
    assert L.fpho_store_create(64, 64, 8, 0, ctypes.byref(h)) == 1
    assert L.fpho_store_create(64, 64, 8, 1, None) == 1
    counts = (ctypes.c_int32 * 1)()
    assert L.fpho_store_count(None, 1, None, None, counts, None) == 1
    assert L.fpho_store_free(None) == 0
    rc = L.fpho_patch_create_device_pixels(None, 1, 0, None, ctypes.byref(h))
    assert rc == 1 and "NULL" in _lib.last_error() and not h.value


def test_new_entry_points_reject_bad_arguments():
    """Host-side checks of the batch configuration, flux-solve, exact-residual
    and variant-shape entry points, made before any CUDA call."""
    from forcepho_b200 import _lib
    L = _lib.lib
    h = ctypes.c_void_p()
    one = (ctypes.c_void_p * 1)(None)
    assert L.fpho_batch_create_config(None, 1, -1, 128, 0, None, ctypes.byref(h)) == 1
    assert L.fpho_batch_create_config(one, 1, -1, 8, 0, None, ctypes.byref(h)) == 1
    assert "live_cap" in _lib.last_error()
    assert L.fpho_batch_create_config(one, 1, -1, 128, 99, None, ctypes.byref(h)) == 1
    assert "ctas_per_sm" in _lib.last_error()
    out = (ctypes.c_int * 16)()
    n = L.fpho_batch_variants(out, 16)
    no_batch = [v for v in range(len(_lib.variants())) if v not in list(out)[:n]][0]
    assert L.fpho_batch_create_config(one, 1, no_batch, 128, 0, None, ctypes.byref(h)) == 1
    assert "no batched tile kernel" in _lib.last_error()
    assert L.fpho_batch_create_config(one, 1, -1, 128, 0, None, ctypes.byref(h)) == 1
    assert "NULL" in _lib.last_error() and not h.value           # the patch itself
    assert n >= 5 and all(out[i] >= 0 for i in range(n))
    assert L.fpho_batch_config(None, out) == 1
    assert L.fpho_patch_optimize_fluxes(None, None, 1, None, None, None, None) == 1
    assert L.fpho_patch_flux_normal_equations(None, None, 1, None, None, None) == 1
    assert L.fpho_patch_set_exact_residual(None, 1) == 1
    shape = (ctypes.c_int * 3)()
    assert L.fpho_variant_shape(-1, shape) == 1 and L.fpho_variant_shape(999, shape) == 1
    assert L.fpho_variant_shape(0, shape) == len(_lib.variants())


def test_fused_posterior_entry_points_reject_bad_arguments():
    """Host-side checks of fpho_build_proposal_bounded and
    fpho_bounded_lnp_grad, made before any CUDA call."""
    from forcepho_b200 import _lib
    L = _lib.get()
    p = ctypes.c_void_p(16)  # never dereferenced: every call below fails its checks first
    assert L.fpho_build_proposal_bounded(None, p, p, p, 1, 1, None, None, None, p, None) == 1
    assert "NULL" in _lib.last_error()
    assert L.fpho_build_proposal_bounded(p, p, p, p, 0, 1, None, None, None, p, None) == 1
    assert L.fpho_build_proposal_bounded(p, p, p, p, 1, 1, p, None, None, p, None) == 1
    assert "together" in _lib.last_error()
    assert L.fpho_build_proposal_bounded(p, p, p, p, 1, 0, None, None, None, p, None) != 0
    assert "n_bands" in _lib.last_error()
    assert L.fpho_bounded_lnp_grad(0, p, p, p, p, p, p, p, 1, p, p, p, 1, p, None) == 1
    assert L.fpho_bounded_lnp_grad(10, None, p, p, p, p, p, p, 1, p, p, p, 1, p, None) == 1
    assert "NULL" in _lib.last_error()
    assert L.fpho_bounded_lnp_grad(600, p, p, p, p, p, p, p, 1, p, p, p, 2, p, None) != 0
    assert "partials" in _lib.last_error()
