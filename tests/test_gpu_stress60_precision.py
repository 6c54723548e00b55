"""GPU: the precision stress patch -- 60 sources (half with sersic in [3.5, 6]
and rh up to 1 arcsec, fluxes LogNormal(0, 3)), 15 bands x 6 exposures of
256x256 px (5.9 M pixels), 6-Gaussian PSFs, 3240 image Gaussians per
exposure.

Checked against the reference CPU kernel (its MAXSOURCES=64 build, band by
band in spawn workers): chi2 relative error <= 1e-6 per band, gradient by the
per-component bar of the parity tests (test_gpu_parity.grad_ok).  Reported
(printed) beside it: the error of this kernel and of the reference against
an all-FP64 evaluation, per band for chi2 and per component for the gradient.
"""
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from test_gpu_parity import grad_ok, res_multiple

pytestmark = pytest.mark.gpu

CHI2_RTOL = 1e-6


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def test_stress60_precision():
    if not O.ref_available(60):
        pytest.skip("reference CPU kernel (64-source build) not built")
    import torch
    from forcepho_b200 import _lib, synth
    from forcepho_b200.proposal import GPUProposer
    P = synth.make_workload("stress60", seed=0, render=synth.render_model_gpu)
    prop = P.proposal()
    nb, ns = P.n_bands, P.n_sources
    P.send_to_device()
    chi2, dchi2 = GPUProposer().evaluate_proposal(prop, patch=P)
    # device-resident timing of the same evaluation
    dp = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    c = torch.zeros(nb, dtype=torch.float64, device="cuda")
    g = torch.zeros(nb * ns * 7, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream()

    def ev():
        _lib.call("fpho_evaluate_proposal", P.device_patch.handle, dp.data_ptr(), ns,
                  c.data_ptr(), g.data_ptr(), 7 * ns, 0, s.cuda_stream)

    for _ in range(3):
        ev()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(10):
        ev()
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 10
    assert torch.equal(c.cpu(), torch.as_tensor(chi2))
    P.free()

    nproc = max(2, min(32, os.cpu_count() or 2))
    with tempfile.TemporaryDirectory() as tmp:
        payload = O.patch_payload_file(P, os.path.join(tmp, "patch.npz"))
        rp = O.ref_pool(ns, nproc)
        op = O.oracle_pool(nproc)
        try:
            ref = rp.starmap(O._worker_eval, [(payload, prop, b) for b in range(nb)])
            f64 = O.f64_many(P, [(prop, b) for b in range(nb)], op, payload)
            mix = O.mixed_abs_many(P, [(prop, b) for b in range(nb)], op, payload)
        finally:
            for p in (rp, op):
                p.close()
                p.join()
    c_ref = np.array([r[1] for r in ref])
    d_ref = np.array([r[2] for r in ref])
    c64 = np.array([c for c, _ in f64])
    d64 = np.array([g for _, g in f64])
    gm = np.array([m[2] for m in mix])
    sc = np.array([m[3] for m in mix])
    rs = np.array([m[5] for m in mix])

    np.testing.assert_allclose(chi2, c_ref, rtol=CHI2_RTOL)
    ok = grad_ok(dchi2, d_ref, gm, sc, rs)
    plain = _rel(dchi2, d_ref) <= 1e-5
    nz = np.abs(d64) > 0
    print(f"60-source patch: {ms:.2f} ms per evaluation on the device "
          f"({P.pairs_per_eval / (ms * 1e-3):.3e} nominal pix-gauss/s)")
    print(f"60-source patch, chi2 rel. error vs FP64: ours max {_rel(chi2, c64).max():.3e}, "
          f"reference max {_rel(c_ref, c64).max():.3e}; ours vs reference max "
          f"{_rel(chi2, c_ref).max():.3e}")
    print(f"60-source patch, gradient rel. error vs FP64 (median / 99th pct / max over "
          f"{int(nz.sum())} components): ours {np.median(_rel(dchi2, d64)[nz]):.2e} / "
          f"{np.percentile(_rel(dchi2, d64)[nz], 99):.2e} / {_rel(dchi2, d64)[nz].max():.2e}; "
          f"reference {np.median(_rel(d_ref, d64)[nz]):.2e} / "
          f"{np.percentile(_rel(d_ref, d64)[nz], 99):.2e} / {_rel(d_ref, d64)[nz].max():.2e}")
    print(f"60-source patch, gradient: {plain.mean():.4f} of components within 1e-5 of the reference; "
          f"largest distance from the exact sum in residual-rounding scales: ours "
          f"{res_multiple(dchi2, gm, rs):.3g}, reference {res_multiple(d_ref, gm, rs):.3g}")
    assert np.all(ok), f"{int((~ok).sum())} gradient components outside the bar"
