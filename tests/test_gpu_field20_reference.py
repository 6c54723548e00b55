"""GPU: the differentiable form on the 20-source, 8-band x 4-exposure,
128x128 px patch against the reference CPU kernel's derivatives on 100
random proposals.

For each proposal theta = truth x (1 + 0.02 N(0, 1)) (q clipped to
[0.3, 1]), d lnlike / d theta comes from the autograd Function and the
per-band dchi2 from the same launch; the reference kernel (oracle/_ref, run
band by band in spawn workers) gives its dchi2 per band.  Bar per component:
relative error <= 1e-5 against the reference, or -- on ill-conditioned
components, where the float reference itself is farther than that from the
exact sum over its own float image Gaussians (the mixed oracle) -- within
max(1e-5 x |mixed|, 2 x the reference's own error, 1e-6 x the sum of
absolute per-pixel contributions, E x the residual-rounding scale) of that
exact sum (test_gpu_parity.grad_ok), E the larger of 4 and the reference's
own worst multiple of that scale over all 100 proposals.  chi2 per band: relative
error <= 1e-6.  The mixed oracle runs only for bands with a component off by
more than 1e-5.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from test_gpu_parity import grad_ok, res_multiple

pytestmark = pytest.mark.gpu

N_PROPOSALS = 100
CHI2_RTOL = 1e-6
GRAD_RTOL = 1e-5


@pytest.fixture(scope="module")
def pools():
    nproc = max(2, min(32, os.cpu_count() or 2))
    print("worker processes:", nproc)
    ref_pool = O.ref_pool(20, nproc) if O.ref_available(20) else None
    orc_pool = O.oracle_pool(nproc)
    yield ref_pool, orc_pool
    for p in (ref_pool, orc_pool):
        if p is not None:
            p.close()
            p.join()


def test_field20_fd_fp64(pools):
    """Central finite differences (h = 1e-4 relative) of the all-FP64 oracle
    on the 20-source patch for one flux per band and all six shape parameters
    of two sources (bar: see fd_check)."""
    from forcepho_b200 import synth
    from forcepho_b200.autograd import PatchEvaluator
    from test_gpu_autograd import fd_check
    P = synth.make_workload("field20", seed=0)
    P.send_to_device()
    ev = PatchEvaluator(P)
    nb, npar = P.n_bands, P.n_bands + 6
    comps = [b * npar + b for b in range(nb)]
    comps += [0 * npar + nb + j for j in range(6)] + [7 * npar + nb + j for j in range(6)]
    for i, g, fd in fd_check(P, ev, P.params, comps, pools[1]):
        print(f"20-source patch, param {i}: autograd {g:.9g} fd {fd:.9g} "
              f"rel {abs(g - fd) / abs(fd):.2e}")
    P.free()


def test_field20_autograd_vs_reference_100_proposals(pools):
    ref_pool, orc_pool = pools
    if ref_pool is None:
        pytest.skip("reference CPU kernel not built")
    import torch
    from forcepho_b200 import synth
    from forcepho_b200.autograd import LnLike, PatchEvaluator
    from forcepho_b200.sources import proposal_from_params
    P = synth.make_workload("field20", seed=0)
    P.send_to_device()
    ev = PatchEvaluator(P)
    nb, ns = P.n_bands, P.n_sources
    rng = np.random.default_rng(42)
    thetas, props, d_gpu, c_gpu, g_auto = [], [], [], [], []
    for k in range(N_PROPOSALS):
        th = P.truth * (1 + 0.02 * rng.standard_normal(P.truth.shape))
        th[:, nb + 2] = np.clip(th[:, nb + 2], 0.3, 1.0)
        t = torch.as_tensor(th, device="cuda").requires_grad_(True)
        ll = LnLike.apply(t, ev)
        ll.backward()
        thetas.append(th)
        props.append(proposal_from_params(th, nb, P.table))
        d_gpu.append(ev.dchi2.cpu().numpy().reshape(nb, ns, 7).astype(np.float64))
        c_gpu.append(ev.chi2.cpu().numpy())
        g_auto.append(t.grad.cpu().numpy())
        # the autograd gradient is the stacked per-band gradient
        st = np.concatenate([d_gpu[-1][:, :, 0].T, d_gpu[-1][:, :, 1:].sum(0)], axis=1)
        np.testing.assert_allclose(g_auto[-1], -0.5 * st, rtol=1e-12, atol=0)
    assert ev.error_word() == 0
    P.free()

    payload = O._patch_payload(P)
    jobs = [(payload, props[k], b) for k in range(N_PROPOSALS) for b in range(nb)]
    res = ref_pool.starmap(O._worker_eval, jobs)
    c_ref = np.zeros((N_PROPOSALS, nb))
    d_ref = np.zeros((N_PROPOSALS, nb, ns, 7))
    for j, (b, c, g, _) in enumerate(res):
        c_ref[j // nb, b], d_ref[j // nb, b] = c, g
    c_gpu = np.array(c_gpu)
    d_gpu = np.array(d_gpu)
    np.testing.assert_allclose(c_gpu, c_ref, rtol=CHI2_RTOL)

    plain = np.abs(d_gpu - d_ref) <= GRAD_RTOL * np.abs(d_ref)
    need = [(k, b) for k in range(N_PROPOSALS) for b in range(nb)
            if not np.all(plain[k, b])]
    mixed = O.mixed_abs_many(P, [(props[k], b) for k, b in need], orc_pool)
    bad, details = 0, []
    worst_ours, worst_ref = 0.0, 0.0
    envelope = max([4.0] + [res_multiple(d_ref[k, b], m[2], m[5])
                            for (k, b), m in zip(need, mixed)])
    for (k, b), (_, _, gm, scale, tscale, rscale) in zip(need, mixed):
        g, r = d_gpu[k, b], d_ref[k, b]
        ok = grad_ok(g, r, gm, scale, rscale, envelope=envelope)
        worst_ours = max(worst_ours, res_multiple(g, gm, rscale))
        worst_ref = max(worst_ref, res_multiple(r, gm, rscale))
        for idx in zip(*np.nonzero(~ok)):
            bad += 1
            details.append((k, b) + tuple(int(i) for i in idx) +
                           (g[idx], r[idx], gm[idx], scale[idx]))
    print(f"20-source patch: {N_PROPOSALS} proposals, fraction of per-band gradient components "
          f"within 1e-5 of the reference: {plain.mean():.4f}; bands needing the "
          f"condition-scale criterion: {len(need)}; failing components: {bad}; "
          f"largest distance from the exact sum in residual-rounding scales: "
          f"ours {worst_ours:.3g}, reference {worst_ref:.3g}")
    for d in details:
        k, b, src, j, g, r, gm, sc = d
        print(f"  proposal {k} band {b} source {src} param {j}: gpu {g:.9g} ref {r:.9g} "
              f"mixed {gm:.9g} |gpu-mixed|/scale {abs(g - gm) / sc:.3g} "
              f"|ref-mixed|/scale {abs(r - gm) / sc:.3g}")
    assert bad == 0
