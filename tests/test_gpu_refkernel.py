"""GPU: the reference's own CUDA kernel (oracle/_ref/librefgpu.so, compiled
from forcepho/src/compute_gaussians_kernel.cu with the reference's options)
on the device copy of a patch -- the GPU baseline of the benchmark.  Its
float arithmetic (device expf, warp-shuffle and atomic reduction order)
differs from the reference CPU kernel's, so it is compared with loose bars:
chi2 relative error <= 1e-5, gradient components within 1e-3 relative or
1e-5 of the band's largest component.  Recorded beside it: how far this
project's kernel and the reference GPU kernel each are from the reference CPU
kernel."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O
from oracle import refgpu

pytestmark = pytest.mark.gpu


def _run_ref_gpu(P, prop):
    import torch
    from forcepho_b200 import _lib
    nb, ns = P.n_bands, P.n_sources
    P.send_to_device()
    dstruct = P.device_patch.device_struct
    dprop = torch.from_numpy(np.ascontiguousarray(prop).view(np.uint8).copy()).cuda()
    chi2 = torch.zeros(nb, dtype=torch.float64, device="cuda")
    resp = torch.zeros(nb * _lib.lib.fpho_sizeof(3) // 4, dtype=torch.float32, device="cuda")
    refgpu.evaluate(dstruct, dprop.data_ptr(), chi2.data_ptr(), resp.data_ptr(), nb, ns,
                    refgpu.max_gauss_band(P), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ms = refgpu.max_sources()
    d = resp.cpu().numpy().reshape(nb, ms, 7)[:, :ns].astype(np.float64)
    P.free()
    return chi2.cpu().numpy(), d


@pytest.mark.parametrize("name", ["single_seed1", "mini_3src_2band"])
def test_reference_gpu_kernel_runs(name):
    if not refgpu.available():
        pytest.skip("reference CUDA kernel not built")
    P, prop, d = load_golden(name)
    c_rg, g_rg = _run_ref_gpu(P, prop)
    from test_gpu_parity import gpu_eval
    c_us, g_us = gpu_eval(P, prop)
    c_ref, g_ref = d["ref_chi2"], d["ref_dchi2"].astype(np.float64)
    np.testing.assert_allclose(c_rg, c_ref, rtol=1e-5)
    tol = np.maximum(1e-3 * np.abs(g_ref), 1e-5 * np.abs(g_ref).max(axis=(1, 2), keepdims=True))
    assert np.all(np.abs(g_rg - g_ref) <= tol)
    rel = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))
    print(f"{name}: vs reference CPU kernel -- chi2: reference GPU {rel(c_rg, c_ref):.2e}, "
          f"ours {rel(c_us, c_ref):.2e}; gradient: reference GPU {rel(g_rg, g_ref):.2e}, "
          f"ours {rel(g_us, g_ref):.2e}")


def test_reference_gpu_kernel_timing_field20():
    """Times the reference CUDA kernel against this project's kernel on the
    20-source, 8-band x 4-exposure, 128x128 px patch (device-resident inputs,
    CUDA events, L2 flushed between evaluations) and checks that the two agree
    (chi2 within 1e-5)."""
    if not refgpu.available():
        pytest.skip("reference CUDA kernel not built")
    import torch
    from forcepho_b200 import _lib, synth
    P = synth.make_workload("field20", seed=0, render=synth.render_model_gpu)
    prop = P.proposal()
    nb, ns = P.n_bands, P.n_sources
    P.send_to_device()
    dstruct = P.device_patch.device_struct
    dprop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    c_rg = torch.zeros(nb, dtype=torch.float64, device="cuda")
    resp = torch.zeros(nb * 210, dtype=torch.float32, device="cuda")
    c_us = torch.zeros(nb, dtype=torch.float64, device="cuda")
    g_us = torch.zeros(nb * ns * 7, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    mg = refgpu.max_gauss_band(P)

    def ref_gpu():
        refgpu.evaluate(dstruct, dprop.data_ptr(), c_rg.data_ptr(), resp.data_ptr(), nb, ns, mg,
                        s.cuda_stream)

    def ours():
        _lib.call("fpho_evaluate_proposal", P.device_patch.handle, dprop.data_ptr(), ns,
                  c_us.data_ptr(), g_us.data_ptr(), 7 * ns, 0, s.cuda_stream)

    def timed(fn, n):
        fn()
        fn()
        ts = []
        for _ in range(n):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    t_ref = timed(ref_gpu, 5)
    t_us = timed(ours, 20)
    np.testing.assert_allclose(c_rg.cpu().numpy(), c_us.cpu().numpy(), rtol=1e-5)
    print(f"20-source patch: reference CUDA kernel {t_ref:.3f} ms per evaluation "
          f"({1e3 / t_ref:.1f} evals/s), this project's {t_us:.3f} ms ({1e3 / t_us:.1f} evals/s): "
          f"{t_ref / t_us:.1f}x")
    P.free()


def test_reference_gpu_kernel_timing_single_and_uneven():
    """Times the reference CUDA kernel on the single-source 64x64 px patch and
    on 256 uneven patches (one launch per patch, as GPUProposer launches it),
    beside this project's plain loop and batched form on the same patches;
    checks agreement of chi2 (1e-5) on every patch."""
    if not refgpu.available():
        pytest.skip("reference CUDA kernel not built")
    import torch
    from forcepho_b200 import _lib, synth
    from forcepho_b200.batch import PatchBatch
    s = torch.cuda.current_stream()

    def setup(P):
        nb, ns = P.n_bands, P.n_sources
        P.send_to_device()
        dprop = torch.from_numpy(P.proposal().view(np.uint8).copy()).cuda()
        return dict(P=P, nb=nb, ns=ns, dstruct=P.device_patch.device_struct, dprop=dprop,
                    mg=refgpu.max_gauss_band(P),
                    c_rg=torch.zeros(nb, dtype=torch.float64, device="cuda"),
                    resp=torch.zeros(nb * 210, dtype=torch.float32, device="cuda"),
                    c_us=torch.zeros(nb, dtype=torch.float64, device="cuda"),
                    g_us=torch.zeros(nb * ns * 7, dtype=torch.float32, device="cuda"))

    def ref_all(items):
        for it in items:
            refgpu.evaluate(it["dstruct"], it["dprop"].data_ptr(), it["c_rg"].data_ptr(),
                            it["resp"].data_ptr(), it["nb"], it["ns"], it["mg"], s.cuda_stream)

    def ours_all(items):
        for it in items:
            _lib.call("fpho_evaluate_proposal", it["P"].device_patch.handle,
                      it["dprop"].data_ptr(), it["ns"], it["c_us"].data_ptr(),
                      it["g_us"].data_ptr(), 7 * it["ns"], 0, s.cuda_stream)

    def timed(fn, n=5):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(n):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    # the single-source patch
    it0 = [setup(synth.make_workload("single", seed=1, render=synth.render_model_gpu))]
    t_ref0, t_us0 = timed(lambda: ref_all(it0), 20), timed(lambda: ours_all(it0), 20)
    np.testing.assert_allclose(it0[0]["c_rg"].cpu().numpy(), it0[0]["c_us"].cpu().numpy(),
                               rtol=1e-5)
    print(f"single-source patch: reference CUDA kernel {t_ref0 * 1e3:.1f} us, "
          f"this project's {t_us0 * 1e3:.1f} us per evaluation")
    it0[0]["P"].free()

    # 256 uneven patches
    patches = synth.make_workload("uneven", seed=3, render=synth.render_model_gpu, n_patches=256)
    items = [setup(P) for P in patches]
    t_ref = timed(lambda: ref_all(items), 3)
    t_us = timed(lambda: ours_all(items), 3)
    for it in items:
        np.testing.assert_allclose(it["c_rg"].cpu().numpy(), it["c_us"].cpu().numpy(),
                                   rtol=1e-5)
    batch = PatchBatch(patches)
    dprop, chi2, dchi2 = batch.device_buffers()
    t_b = timed(lambda: batch.evaluate_device(dprop, chi2, dchi2), 5)
    nominal = sum(P.pairs_per_eval for P in patches)
    print(f"256 uneven patches: reference CUDA kernel {t_ref:.2f} ms "
          f"({256 / (t_ref * 1e-3):.0f} patch-evals/s, {nominal / (t_ref * 1e-3):.3e} "
          f"pix-gauss/s); this project's plain loop {t_us:.2f} ms; batched {t_b:.2f} ms "
          f"({256 / (t_b * 1e-3):.0f} patch-evals/s, {nominal / (t_b * 1e-3):.3e} pix-gauss/s)")
    batch.free()
    for P in patches:
        P.free()
