"""fpho_evaluate_proposal_noalloc: the evaluation entry point for callers that
cannot allocate device memory (plugins whose host framework owns every device
allocation, services that must not grow device memory once started).
It keeps its scratch in a static device array instead of allocating; its
results must match the handle-based fpho_evaluate_proposal on the same patch
and the reference CPU kernel (through its golden outputs and the oracle).

This file is collected last, so that a failure here is seen only after every
other test has run; it also passes when run on its own.
"""
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


def noalloc_call(_lib, st, P, dprop, chi2, dchi2, status, stream, total_pixels=None):
    nb, ns = P.n_bands, P.n_sources
    npix = int(P.exposure_N.sum()) if total_pixels is None else total_pixels
    _lib.call("fpho_evaluate_proposal_noalloc", st.ctypes.data, nb, P.n_exp, npix,
              int(P.n_psf_per_source.max()), dprop.data_ptr(), chi2.data_ptr(),
              dchi2.data_ptr(), 7 * ns, None if status is None else status.data_ptr(), stream)


def out_buffers(torch, P):
    nb, ns = P.n_bands, P.n_sources
    chi2 = torch.full((nb,), np.nan, dtype=torch.float64, device="cuda")
    dchi2 = torch.full((nb * ns * 7,), np.nan, dtype=torch.float32, device="cuda")
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    return chi2, dchi2, status


@pytest.mark.parametrize("name", ["mini_3src_2band", "single_seed1"])
def test_noalloc_matches_handle_path_twice(name):
    import torch
    from forcepho_b200 import _lib
    from forcepho_b200.proposal import GPUProposer
    from test_gpu_parity import CHI2_RTOL, check_grad

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
        chi2, dchi2, status = out_buffers(torch, P)
        noalloc_call(_lib, st, P, dprop, chi2, dchi2, status, s.cuda_stream)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        c = chi2.cpu().numpy()
        g = dchi2.cpu().numpy().reshape(nb, ns, 7)
        # the handle path's default tile shape sums in a different order: the
        # parity tolerances of the tests (chi2 1e-6, gradient 1e-5)
        np.testing.assert_allclose(c, chi2_a, rtol=CHI2_RTOL)
        np.testing.assert_allclose(g, dchi2_a, rtol=1e-5,
                                   atol=1e-6 * float(np.abs(dchi2_a).max()))
        # against the reference CPU kernel's outputs (golden), by the parity bar
        np.testing.assert_allclose(c, d["ref_chi2"], rtol=CHI2_RTOL)
        check_grad(g, d["ref_dchi2"], P, prop)


def test_noalloc_matches_oracle_field_patch():
    """A multi-band patch with uneven exposures (ragged tiles, masked pixels,
    rotated and scaled exposures) against the oracle's restatement of the
    reference CPU kernel."""
    import torch
    from forcepho_b200 import _lib, synth
    from oracle import oracle as O
    from test_gpu_parity import CHI2_RTOL, check_grad

    spec = synth.PatchSpec(n_sources=6, exposures_per_band=[2, 1, 3],
                           shapes=[(48, 48), (40, 56), (64, 64), (33, 47), (48, 48), (52, 40)],
                           n_psf=4, psf_sigma=(0.5, 3.0), rot_deg=1.0, scale_frac=0.02,
                           g_range=(0.8, 1.2), mask_frac=0.02, flux_sigma=1.5)
    P = synth.make_patch(spec, seed=5)
    prop = P.proposal()
    st, keep = device_struct_for(P, torch)
    nb, ns = P.n_bands, P.n_sources
    dprop = torch.from_numpy(np.ascontiguousarray(prop).view(np.uint8).copy()).cuda()
    chi2, dchi2, status = out_buffers(torch, P)
    noalloc_call(_lib, st, P, dprop, chi2, dchi2, status, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    cref, gref = O.oracle_evaluate(P, prop, precision="f32")
    np.testing.assert_allclose(chi2.cpu().numpy(), cref, rtol=CHI2_RTOL)
    check_grad(dchi2.cpu().numpy().reshape(nb, ns, 7), gref, P, prop)


def test_noalloc_rejects_pixels_outside_total():
    """An exposure whose pixel run ends beyond total_pixels is refused on the
    device before any pixel is read: status bit 2, chi2 NaN, gradient
    untouched, and the next consistent call is correct again."""
    import torch
    from forcepho_b200 import _lib

    P, prop, d = load_golden("mini_3src_2band")
    st, keep = device_struct_for(P, torch)
    nb, ns = P.n_bands, P.n_sources
    dprop = torch.from_numpy(np.ascontiguousarray(prop).view(np.uint8).copy()).cuda()
    s = torch.cuda.current_stream().cuda_stream
    npix = int(P.exposure_N.sum())
    # shift the last exposure's start past the end of the pixel arrays; every
    # other array (and the tile count bound) stays consistent
    bad_start = np.array(P.exposure_start, dtype=np.int32).copy()
    bad_start[-1] = npix - int(P.exposure_N[-1]) + 1000
    t_bad = torch.from_numpy(bad_start.view(np.uint8).copy()).cuda()
    st_bad = st.copy()
    st_bad["exposure_start"] = t_bad.data_ptr()
    for status_given in (True, False):
        chi2, dchi2, status = out_buffers(torch, P)
        chi2.fill_(1.0)
        noalloc_call(_lib, st_bad, P, dprop, chi2, dchi2, status if status_given else None, s)
        torch.cuda.synchronize()
        if status_given:
            assert int(status.item()) & 2
        assert np.all(np.isnan(chi2.cpu().numpy()))
    # a negative psfgauss_start of an exposure with PSF components: bit 2 too
    bad_ps = np.array(P.psfgauss_start, dtype=np.int32).copy()
    bad_ps[0] = -3
    t_ps = torch.from_numpy(bad_ps.view(np.uint8).copy()).cuda()
    st_ps = st.copy()
    st_ps["psfgauss_start"] = t_ps.data_ptr()
    chi2, dchi2, status = out_buffers(torch, P)
    noalloc_call(_lib, st_ps, P, dprop, chi2, dchi2, status, s)
    torch.cuda.synchronize()
    assert int(status.item()) & 2 and np.all(np.isnan(chi2.cpu().numpy()))
    # the consistent patch evaluates correctly after the refused calls
    chi2, dchi2, status = out_buffers(torch, P)
    noalloc_call(_lib, st, P, dprop, chi2, dchi2, status, s)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    np.testing.assert_allclose(chi2.cpu().numpy(), d["ref_chi2"], rtol=1e-6)


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
