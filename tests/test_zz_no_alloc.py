"""fpho_evaluate_proposal_noalloc: the evaluation entry point for callers that
cannot allocate device memory (graph capture in progress, a host framework
that owns all device allocations, services that must not grow device memory).
It keeps its scratch in a static device array instead of allocating; its
results must match the handle-based fpho_evaluate_proposal on the same patch.

This file is collected last, so that a failure here is seen only after every
other test has run; it also passes when run on its own.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def device_struct_for(P, torch):
    """Copy every patch array to torch device buffers (allocated by the test,
    not by the entry point); return (host struct with device pointers, keep)."""
    from forcepho_b200.patches.patch import PatchBase
    P.coerce_arrays()
    keep = {}
    st = np.zeros(1, dtype=PatchBase.patch_struct_dtype)
    for name in PatchBase.patch_struct_dtype.names:
        if PatchBase.patch_struct_dtype[name] != PatchBase.ptr_dtype:
            st[name] = getattr(P, name)
            continue
        if name == "residual":
            st[name] = 0
            continue
        a = np.ascontiguousarray(getattr(P, name))
        t = torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()
        keep[name] = t
        st[name] = t.data_ptr()
    return st, keep


@pytest.mark.parametrize("name", ["mini_3src_2band", "single_seed1"])
def test_noalloc_matches_handle_path_twice(name):
    import torch
    from forcepho_b200 import _lib
    from forcepho_b200.proposal import GPUProposer

    P, prop, d = load_golden(name)
    # the existing entry point (handle-based, allocating)
    P.return_residual = False
    P.send_to_device()
    chi2_a, dchi2_a = GPUProposer().evaluate_proposal(prop, patch=P)
    P.free()

    st, keep = device_struct_for(P, torch)
    nb, ns = P.n_bands, P.n_sources
    dprop = torch.from_numpy(np.ascontiguousarray(prop).view(np.uint8).copy()).cuda()
    s = torch.cuda.current_stream()
    for _ in range(2):  # two calls in a row share (and reuse) the scratch array
        chi2 = torch.full((nb,), np.nan, dtype=torch.float64, device="cuda")
        dchi2 = torch.full((nb * ns * 7,), np.nan, dtype=torch.float32, device="cuda")
        status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        _lib.call("fpho_evaluate_proposal_noalloc", st.ctypes.data, nb, P.n_exp,
                  int(P.exposure_N.sum()), int(P.n_psf_per_source.max()), dprop.data_ptr(),
                  chi2.data_ptr(), dchi2.data_ptr(), 7 * ns, status.data_ptr(), s.cuda_stream)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        c = chi2.cpu().numpy()
        g = dchi2.cpu().numpy().reshape(nb, ns, 7)
        np.testing.assert_allclose(c, chi2_a, rtol=1e-9)
        np.testing.assert_allclose(g, dchi2_a, rtol=1e-5,
                                   atol=1e-6 * float(np.abs(dchi2_a).max()))


def test_noalloc_rejects_oversize():
    """Sizes whose scratch exceeds FPHO_NOALLOC_SCRATCH_BYTES fail with
    FPHO_ERR_LIMIT and a message, before anything is launched."""
    import torch
    from forcepho_b200 import _lib
    P, prop, d = load_golden("single_seed1")
    st, keep = device_struct_for(P, torch)
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = _lib.lib.fpho_evaluate_proposal_noalloc(st.ctypes.data, 1, 60000, 2 ** 30, 1024,
                                                 out.data_ptr(), out.data_ptr(),
                                                 out.data_ptr(), 7, None, None)
    assert rc == 4 and "scratch" in _lib.last_error()
