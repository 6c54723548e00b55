"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Tolerances (the bar stated for this path):
  * chi2: relative error <= 1e-6 against the reference CPU kernel.
  * gradient, per component: relative error <= 1e-5 against the reference
    CPU kernel; on ill-conditioned components, where the reference itself is
    farther than 1e-5 from the exact sum over its own float image Gaussians
    (the "mixed" oracle: the reference's float Gaussians, FP64 pixel
    arithmetic and sums), no farther from that exact sum than the largest of
    twice the reference's own distance, 1e-6 of the sum of absolute per-pixel
    contributions, and 4x the residual-rounding scale (how far a float
    rounding of the residual r alone moves the component, summed over pixels),
    or the reference's own worst multiple of that scale on the same
    evaluation if larger (it reaches 18-20x on the 20- and 60-source patches).  The distance of both float kernels
    from an all-FP64 evaluation (float image-Gaussian centres carry ~4e-6 px
    of rounding) is reported, not asserted tightly.
  * image Gaussians: bit-identical to the reference's.
  * residual image: |gpu - ref| <= 1e-5 * max|data| per pixel.
"""
import ctypes

import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CHI2_RTOL = 1e-6
GRAD_RTOL = 1e-5
# Number of compiled tile kernels (tests/test_abi.py checks the library's count).
N_VARIANTS = 14


def gpu_eval(P, prop, residual=False, variant=None, live_cap=None):
    from forcepho_b200.proposal import GPUProposer
    P.return_residual = residual
    P.free()
    P.send_to_device()
    if variant is not None:
        P.device_patch.set_config(variant, live_cap or 512)
    out = GPUProposer().evaluate_proposal(prop, patch=P, unpack=False)
    P.free()
    return out


def grad_report(g, ref, f64, mixed):
    g, ref, f64, mixed = (np.asarray(a, dtype=np.float64) for a in (g, ref, f64, mixed))
    rel = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))
    return {"gpu_vs_ref": rel(g, ref), "gpu_vs_mixed": rel(g, mixed),
            "gpu_vs_fp64": rel(g, f64), "ref_vs_fp64": rel(ref, f64)}


ABS_RTOL = 1e-6
RES_SCALE = 4.0


def res_multiple(x, mixed, rscale):
    """Largest |x - mixed| / rscale over components with rscale > 0."""
    d = np.abs(np.asarray(x, np.float64) - mixed)
    r = np.asarray(rscale, np.float64)
    return float(np.max(np.where(r > 0, d / np.where(r > 0, r, 1.0), 0.0), initial=0.0))


def grad_ok(g, ref, mixed, scale, rscale, rtol=GRAD_RTOL, envelope=None):
    """The per-component bar (arrays of equal shape): within rtol of the
    reference CPU kernel, or within max(rtol |mixed|, 2 |ref - mixed|,
    ABS_RTOL scale, E rscale) of the exact sum `mixed`, where E is the larger of
    RES_SCALE and the reference's own largest |ref - mixed| / rscale over the
    arrays given (or `envelope`): no component farther from the exact sum, in
    residual-rounding scales, than the reference's worst."""
    g, ref = (np.asarray(a, dtype=np.float64) for a in (g, ref))
    own = np.abs(ref - mixed)
    if envelope is None:
        envelope = max(RES_SCALE, res_multiple(ref, mixed, rscale))
    return (np.abs(g - ref) <= rtol * np.abs(ref)) | \
        (np.abs(g - mixed) <= np.maximum.reduce([rtol * np.abs(mixed), 2.0 * own,
                                                 ABS_RTOL * scale, envelope * rscale]))


def check_grad(g, ref, P, prop, rtol=GRAD_RTOL):
    """Per component: within rtol of the reference CPU kernel; or, on an
    ill-conditioned component (where the float reference is itself off the
    exact value by more than rtol), within the condition-scale allowance of
    ``grad_ok`` of the exact sum over the reference's float image Gaussians.
    Returns the fraction meeting the plain bar."""
    _, mixed, scale, _, rscale = O.oracle_mixed_abs(P, prop, terms=True)
    g, ref = (np.asarray(a, dtype=np.float64) for a in (g, ref))
    ok = grad_ok(g, ref, mixed, scale, rscale, rtol)
    bad = ~ok
    assert np.all(ok), (f"{bad.sum()} components: gpu {g[bad]}, ref {ref[bad]}, "
                        f"mixed {mixed[bad]}, scale {scale[bad]}")
    return float(np.mean(np.abs(g - ref) <= rtol * np.abs(ref)))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_parity(name):
    P, prop, d = load_golden(name)
    chi2, dchi2 = gpu_eval(P, prop)
    np.testing.assert_allclose(chi2, d["ref_chi2"], rtol=CHI2_RTOL)
    c64, g64 = O.oracle_evaluate(P, prop, precision="f64")
    cm, gm = O.oracle_evaluate(P, prop, precision="mixed")
    np.testing.assert_allclose(chi2, c64, rtol=CHI2_RTOL)
    print(name, grad_report(dchi2, d["ref_dchi2"], g64, gm))
    frac = check_grad(dchi2, d["ref_dchi2"], P, prop)
    print(name, "fraction within 1e-5 of the reference:", frac)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_vs_slow_fp64(name):
    """Against the reference's FP64 slow path (no cutoff): the cutoff changes
    chi2 by < 1e-6 relative on these patches."""
    P, prop, d = load_golden(name)
    chi2, dchi2 = gpu_eval(P, prop)
    np.testing.assert_allclose(chi2, d["slow_chi2"], rtol=2e-6)
    np.testing.assert_allclose(dchi2, d["slow_dchi2"], rtol=5e-4,
                               atol=1e-6 * np.abs(d["slow_dchi2"]).max())


def test_residual_matches_oracle():
    P, prop, d = load_golden("mini_3src_2band")
    chi2, dchi2, res = gpu_eval(P, prop, residual=True)
    c, g, r = O.oracle_evaluate(P, prop, residual=True)
    scale = np.abs(P.data).max()
    assert np.max(np.abs(res - r)) <= 1e-5 * scale


@pytest.mark.parametrize("variant", range(N_VARIANTS))
@pytest.mark.parametrize("live_cap", [32, 160])
def test_variants_agree(variant, live_cap):
    """Every compiled tile shape (classic and Gaussian-split) against the
    reference; live_cap 32 forces several staged chunks per tile."""
    P, prop, d = load_golden("mini_3src_2band")
    chi2, dchi2 = gpu_eval(P, prop, variant=variant, live_cap=live_cap)
    c64, g64 = O.oracle_evaluate(P, prop, precision="f64")
    cm, gm = O.oracle_evaluate(P, prop, precision="mixed")
    np.testing.assert_allclose(chi2, c64, rtol=CHI2_RTOL)
    check_grad(dchi2, d["ref_dchi2"], P, prop)


def test_multi_chunk_staging():
    """live_cap smaller than the kept Gaussians forces several staged chunks."""
    from forcepho_b200 import synth
    spec = synth.workload_spec("field20")
    spec.shapes = [(48, 48)] * 32
    P = synth.make_patch(spec, seed=4)
    prop = P.proposal()
    a = gpu_eval(P, prop, variant=1, live_cap=128)  # 128 threads, 128 records per chunk
    b = gpu_eval(P, prop, variant=1, live_cap=1024)
    c64, g64 = O.oracle_evaluate(P, prop, precision="f64")
    np.testing.assert_allclose(a[0], c64, rtol=CHI2_RTOL)
    np.testing.assert_allclose(b[0], c64, rtol=CHI2_RTOL)
    np.testing.assert_allclose(a[1], b[1], rtol=1e-5, atol=1e-6 * np.abs(g64).max())


def test_deterministic():
    P, prop, d = load_golden("mini_3src_2band")
    a = gpu_eval(P, prop)
    b = gpu_eval(P, prop)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_reference_kernel_argument_list():
    """fpho_EvaluateProposal takes the reference kernel's arguments (device
    Patch*, Source*, double*, Response*)."""
    import torch
    from forcepho_b200 import _lib
    from forcepho_b200.proposal import response_struct_dtype
    P, prop, d = load_golden("mini_3src_2band")
    P.return_residual = False
    P.send_to_device()
    dp = P.device_patch
    dprop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    chi2 = torch.zeros(P.n_bands, dtype=torch.float64, device="cuda")
    resp = torch.zeros(P.n_bands * response_struct_dtype.itemsize // 4, dtype=torch.float32,
                       device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    _lib.call("fpho_EvaluateProposal", dp.handle, dp.device_struct, dprop.data_ptr(),
              chi2.data_ptr(), resp.data_ptr(), s)
    torch.cuda.synchronize()
    g = resp.cpu().numpy().reshape(P.n_bands, 30, 7)
    np.testing.assert_allclose(chi2.cpu().numpy(), d["ref_chi2"], rtol=CHI2_RTOL)
    assert np.all(g[:, P.n_sources:] == 0)
    c64, g64 = O.oracle_evaluate(P, prop, precision="f64")
    cm, gm = O.oracle_evaluate(P, prop, precision="mixed")
    check_grad(g[:, :P.n_sources], d["ref_dchi2"], P, prop)
    with pytest.raises(_lib.FphoError):
        _lib.call("fpho_EvaluateProposal", dp.handle, dp.device_struct + 8, dprop.data_ptr(),
                  chi2.data_ptr(), resp.data_ptr(), s)
    P.free()


def test_swap_on_device_invariant():
    """After swap_on_device the residual becomes the data; evaluating the same
    proposal again gives residual_new == data - 2 model (tests/cswap_test.py:98-110
    of the reference)."""
    P, prop, d = load_golden("mini_3src_2band")
    P.return_residual = True
    P.send_to_device()
    from forcepho_b200.proposal import GPUProposer
    pr = GPUProposer()
    _, _, r1 = pr.evaluate_proposal(prop, patch=P, unpack=False)
    P.swap_on_device()
    data_now = P.retrieve_array("data")
    np.testing.assert_array_equal(data_now, r1)
    _, _, r2 = pr.evaluate_proposal(prop, patch=P, unpack=False)
    model = P.data - r1
    np.testing.assert_allclose(r2, P.data - 2 * model, atol=1e-5 * np.abs(P.data).max())
    P.free()


def test_field20_full_size():
    """The 20-source patch at full size against FP64 and the reference kernel."""
    from forcepho_b200 import synth
    P = synth.make_workload("field20", seed=0)
    prop = P.proposal()
    chi2, dchi2 = gpu_eval(P, prop)
    c64, g64 = O.oracle_evaluate(P, prop, precision="f64")
    cm, gm = O.oracle_evaluate(P, prop, precision="mixed")
    rc, rd = O.ref_evaluate(P, prop)
    np.testing.assert_allclose(chi2, rc, rtol=CHI2_RTOL)
    np.testing.assert_allclose(chi2, c64, rtol=CHI2_RTOL)
    print("20-source patch", grad_report(dchi2, rd, g64, gm))
    frac = check_grad(dchi2, rd, P, prop)
    print("20-source patch: fraction within 1e-5 of the reference:", frac)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_image_gaussians_bitexact(name):
    """The image Gaussians (centre, inverse covariance, amplitude) built on
    the device equal the reference CPU kernel's float values bit for bit."""
    import ctypes
    from forcepho_b200 import _lib
    P, prop, d = load_golden(name)
    P.return_residual = False
    P.send_to_device()
    from forcepho_b200.proposal import GPUProposer
    GPUProposer().evaluate_proposal(prop, patch=P)
    n_exact = n_total = 0
    for b in range(P.n_bands):
        for e in range(int(P.band_start[b]), int(P.band_start[b] + P.band_N[b])):
            ref = O.image_gaussians_f32(P, prop, b, e)
            buf = np.zeros((len(ref), 32), dtype=np.float32)
            n = ctypes.c_int()
            _lib.call("fpho_patch_image_gaussians", P.device_patch.handle, e, buf.ctypes.data,
                      len(ref), ctypes.byref(n))
            assert n.value == len(ref)
            # reference ImageGaussian order: amp, xcen, ycen, fxx, fyy, fxy
            got = np.stack([buf[:, 10], -buf[:, 0], -buf[:, 2], buf[:, 4], buf[:, 8], buf[:, 6]],
                           1)
            want = ref[:, :6]
            np.testing.assert_array_equal(got, want)
            n_exact += got.size
            n_total += got.size
    P.free()
    assert n_exact == n_total


def test_field20_every_shape():
    """The 20-source patch at full size through every compiled tile shape
    (classic and Gaussian-split), one CTA per tile and persistent, against
    the reference kernel by the per-component bar."""
    from forcepho_b200 import _lib, synth
    from forcepho_b200.proposal import GPUProposer
    P = synth.make_workload("field20", seed=0)
    prop = P.proposal()
    rc, rd = O.ref_evaluate(P, prop)
    _, mixed, scale, _, rscale = O.oracle_mixed_abs(P, prop, terms=True)
    P.return_residual = False
    P.send_to_device()
    for v in range(len(_lib.variants())):
        for sched in (0, 1):
            P.device_patch.set_config(v, 160)
            P.device_patch.set_schedule(sched)
            for _ in range(2):   # the second persistent evaluation follows the first's costs
                chi2, dchi2 = GPUProposer().evaluate_proposal(prop, patch=P)
            np.testing.assert_allclose(chi2, rc, rtol=CHI2_RTOL)
            ok = grad_ok(dchi2, rd, mixed, scale, rscale)
            assert np.all(ok), (v, sched, int((~ok).sum()))
    P.free()


@pytest.mark.parametrize("variant", [3, 6, 0, 8, 10])
def test_persistent_schedule_identical(variant):
    """The persistent schedule (tiles taken by decreasing cost of the previous
    evaluation, through an atomic counter) gives bit-identical chi2 and
    gradients to one CTA per tile -- on the first evaluation (no costs yet)
    and on later ones, with the proposal changing in between."""
    import torch
    from forcepho_b200 import _lib, synth
    P = synth.make_workload("field20", seed=5)
    P.send_to_device()
    h = P.device_patch.handle
    nb, ns = P.n_bands, P.n_sources
    props = [P.proposal(), P.truth_proposal(), P.proposal()]
    c = torch.zeros(nb, dtype=torch.float64, device="cuda")
    g = torch.zeros(nb * ns * 7, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    out = {}
    for sched in (0, 1):
        P.device_patch.set_config(variant, 192)
        P.device_patch.set_schedule(sched)
        res = []
        for q in props:
            dq = torch.from_numpy(q.view(np.uint8).copy()).cuda()
            _lib.call("fpho_evaluate_proposal", h, dq.data_ptr(), ns, c.data_ptr(), g.data_ptr(),
                      7 * ns, 0, s)
            torch.cuda.synchronize()
            res.append((c.clone(), g.clone()))
        out[sched] = res
    for (c0, g0), (c1, g1) in zip(out[0], out[1]):
        assert torch.equal(c0, c1)
        assert torch.equal(g0, g1)
    w = ctypes.c_int()
    _lib.call("fpho_patch_error_word", h, ctypes.byref(w))
    assert w.value == 0
    P.free()
