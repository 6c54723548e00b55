"""GPU: proposals built on the device, the chi2-only kernel, the
differentiable form (torch.autograd.Function), the device posterior and the
graph-captured leapfrog.

Tolerances:
  * device splines vs scipy RectBivariateSpline: |diff| <= 1e-12 x max|coef|
    (value) and 1e-10 x max|coef| (derivatives), both evaluated in FP64;
  * device proposal vs the host proposal (scipy, then float32): equal up to
    one float32 ulp per field;
  * chi2-only chi2 == full chi2, bit for bit (pass 1 is shared);
  * autograd gradient vs central finite differences of the all-FP64 oracle
    (h = 1e-4 relative; see fd_check): relative error <= 1e-4 per component,
    or 1e-6 of the component's sum of absolute per-pixel contributions (the
    float32 kernel is ~1e-5 from FP64; the FD truncation error is < 1e-6);
  * autograd gradient vs the reference kernel's derivatives on 100 random
    proposals: the per-component bar of the parity tests (1e-5 relative, or
    the condition-scale criterion on ill-conditioned components);
  * leapfrog: graph replay == eager loop bit for bit; the energy error over
    a fixed trajectory length shrinks 3-5x when the step is halved (second
    order), which holds only if the gradient is the derivative of lnp.
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-5


def _torch():
    import torch
    return torch


def _f32_round(x):
    return np.asarray(x, dtype=np.float64).astype(np.float32).astype(np.float64)


# ------------------------------------------------------------------ splines
def test_spline_points_match_scipy():
    from forcepho_b200.device_proposal import DeviceSersicTable
    from forcepho_b200.sources import default_table
    T = default_table()
    D = DeviceSersicTable(T)
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(0.5, 6.6, 300), [0.8, 6.2, 7.0, 0.6, 3.0]])
    y = np.concatenate([rng.uniform(-0.05, 1.2, 300), [0.0, 1.0, 0.5, 0.5, 1.5]])
    out = D.points(x, y).cpu().numpy()
    _, _, c = T.knots_and_coeffs()
    for k in range(T.n_radii):
        sp = T.splines[k]
        scale = np.abs(c[k]).max()
        v = np.array([sp(a, b)[0, 0] for a, b in zip(x, y)])
        vx = np.array([sp(a, b, dx=1)[0, 0] for a, b in zip(x, y)])
        vy = np.array([sp(a, b, dy=1)[0, 0] for a, b in zip(x, y)])
        assert np.max(np.abs(out[:, k, 0] - v)) <= 1e-12 * scale
        assert np.max(np.abs(out[:, k, 1] - vx)) <= 1e-10 * scale
        assert np.max(np.abs(out[:, k, 2] - vy)) <= 1e-10 * scale
    D.free()


def _ulp_close(a, b, n=1):
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7fffffff), ia)
    ib = np.where(ib < 0, -(ib & 0x7fffffff), ib)
    return np.all(np.abs(ia - ib) <= n)


def test_build_proposal_matches_host():
    torch = _torch()
    from forcepho_b200 import synth
    from forcepho_b200.device_proposal import DeviceSersicTable, proposal_bytes_to_struct
    from forcepho_b200.sources import proposal_from_params
    P = synth.make_workload("field20", seed=2)
    params = P.params.copy()
    params[0, P.n_bands + 4] = 0.5      # sersic below the table: one-hot nearest radius
    params[1, P.n_bands + 5] = -0.01    # rh < 0: one-hot radius 0
    params[2, P.n_bands + 4] = 6.5      # sersic above the table: FITPACK clamps
    D = DeviceSersicTable(P.table)
    dev = D.build_proposal(torch.as_tensor(params, device="cuda"), P.n_bands)
    got = proposal_bytes_to_struct(dev)
    want = proposal_from_params(params, P.n_bands, P.table)
    for f in want.dtype.names:
        assert _ulp_close(got[f], want[f]), f
    D.free()


# ------------------------------------------------------------------ chi2-only kernel
def test_chi2_only_matches_full():
    torch = _torch()
    from forcepho_b200 import synth
    from forcepho_b200.autograd import PatchEvaluator
    P = synth.make_workload("field20", seed=0)
    P.send_to_device()
    ev = PatchEvaluator(P)
    theta = torch.as_tensor(P.params, device="cuda")
    ev.run(theta, grad=True)
    full = ev.chi2.clone()
    ev.chi2.zero_()
    ev.run(theta, grad=False)
    torch.cuda.synchronize()
    assert torch.equal(full, ev.chi2)
    assert ev.error_word() == 0
    P.free()


# ------------------------------------------------------------------ autograd
def _lnlike_f64(P, theta):
    from forcepho_b200.sources import proposal_from_params
    prop = proposal_from_params(theta, P.n_bands, P.table)
    c, _ = O.oracle_evaluate(P, prop, precision="f64")
    return -0.5 * c.sum()


def _autograd_grad(ev, theta):
    torch = _torch()
    from forcepho_b200.autograd import LnLike
    t = torch.as_tensor(theta, device="cuda").clone().requires_grad_(True)
    ll = LnLike.apply(t, ev)
    ll.backward()
    return float(ll.detach()), t.grad.cpu().numpy().reshape(-1)


def _amps_f64(table, theta, n_bands):
    """(n_sources, 10) float64 mixture amplitudes of theta (Scene order)."""
    p = np.asarray(theta).reshape(-1, n_bands + 6)
    out = np.zeros((len(p), 10))
    for i, row in enumerate(p):
        out[i, :table.n_radii] = table.amplitudes(row[n_bands + 4], row[n_bands + 5])
    return out


def fd_check(P, ev, theta, comps, pool, h=1e-4):
    """Autograd d lnlike / d theta against central finite differences of the
    all-FP64 oracle's lnlike, step h relative, for the flat parameter indices
    ``comps``.

    The proposal holds float32, so steps in flux, ra, dec, q and pa go
    between float32-representable values; steps in sersic and rh act only
    through the mixture amplitudes, which the FP64 oracle then takes in
    double from the splines (float32 amplitudes would put ~2e-4 of rounding
    noise into an h = 1e-4 difference).  Bar: |g - fd| <= max(1e-4 |fd|,
    1e-6 x the sum of absolute per-pixel contributions to the component).
    Returns [(index, g, fd)]."""
    from forcepho_b200.sources import proposal_from_params
    nb, ns = P.n_bands, P.n_sources
    npar = nb + 6
    theta = _f32_round(np.asarray(theta).reshape(-1))
    _, g = _autograd_grad(ev, theta.reshape(ns, npar))
    prop0 = proposal_from_params(theta, nb, P.table)
    dabs = np.zeros((nb, ns, 7))
    mixed = O.mixed_abs_many(P, [(prop0, b) for b in range(nb)], pool)
    for b, (_, _, _, a, _, _) in enumerate(mixed):
        dabs[b] = a
    scale = 0.5 * np.concatenate([dabs[:, :, 0].T, dabs[:, :, 1:].sum(0)], axis=1).reshape(-1)
    jobs, plan = [], []
    for i in comps:
        j = i % npar
        bands = [j] if j < nb else list(range(nb))
        tp, tm = theta.copy(), theta.copy()
        if j >= nb + 4:
            tp[i], tm[i] = theta[i] * (1 + h), theta[i] * (1 - h)
            ap, am = _amps_f64(P.table, tp, nb), _amps_f64(P.table, tm, nb)
            jobs += [(prop0, b, ap) for b in bands] + [(prop0, b, am) for b in bands]
        else:
            tp[i] = _f32_round(theta[i] * (1 + h))
            tm[i] = _f32_round(theta[i] * (1 - h))
            pp = proposal_from_params(tp, nb, P.table)
            pm = proposal_from_params(tm, nb, P.table)
            jobs += [(pp, b) for b in bands] + [(pm, b) for b in bands]
        plan.append((i, len(bands), tp[i] - tm[i]))
    chi = O.f64_chi2_many(P, jobs, pool)
    out, o = [], 0
    for i, n, den in plan:
        fd = -0.5 * (sum(chi[o:o + n]) - sum(chi[o + n:o + 2 * n])) / den
        o += 2 * n
        tol = max(1e-4 * abs(fd), 1e-6 * scale[i])
        assert abs(g[i] - fd) <= tol, (i, g[i], fd, scale[i])
        out.append((i, g[i], fd))
    return out


@pytest.fixture(scope="module")
def oracle_workers():
    import os
    pool = O.oracle_pool(max(2, min(32, os.cpu_count() or 2)))
    yield pool
    pool.close()
    pool.join()


@pytest.mark.parametrize("mode", ["fused", "recompute"])
def test_autograd_vs_fd_fp64_single(mode, oracle_workers):
    from forcepho_b200 import synth
    from forcepho_b200.autograd import PatchEvaluator
    P = synth.make_workload("single", seed=3)
    P.send_to_device()
    ev = PatchEvaluator(P, mode=mode)
    res = fd_check(P, ev, P.params, range(P.n_bands + 6), oracle_workers)
    for i, g, fd in res:
        print(f"single-source patch [{mode}] param {i}: autograd {g:.9g} fd {fd:.9g} "
              f"rel {abs(g - fd) / abs(fd):.2e}")
    P.free()


def test_recompute_equals_fused():
    torch = _torch()
    from forcepho_b200 import synth
    from forcepho_b200.autograd import PatchEvaluator
    P = synth.make_workload("field20", seed=1)
    P.send_to_device()
    a = PatchEvaluator(P, mode="fused")
    b = PatchEvaluator(P, mode="recompute")
    la, ga = _autograd_grad(a, P.params)
    lb, gb = _autograd_grad(b, P.params)
    assert la == lb
    assert np.array_equal(ga, gb)
    P.free()


def test_autograd_vs_reference_single_100_proposals():
    """d lnlike / d theta from the autograd Function against the reference
    kernel's derivatives, stacked as FastPosterior.stack_grad does, on 100
    random proposals around the truth."""
    from forcepho_b200 import synth
    from forcepho_b200.autograd import PatchEvaluator
    from forcepho_b200.model import FastPosterior, BoundedTransform
    from forcepho_b200.sources import proposal_from_params
    if not O.ref_available(1):
        pytest.skip("reference CPU kernel not built")
    P = synth.make_workload("single", seed=11)
    P.send_to_device()
    ev = PatchEvaluator(P)
    fp = FastPosterior(None, P, scene=object(), transform=BoundedTransform([0], [1]))
    rng = np.random.default_rng(0)
    nb = P.n_bands
    fracs = []
    for k in range(100):
        theta = P.truth * (1 + 0.02 * rng.standard_normal(P.truth.shape))
        theta[:, nb + 2] = np.clip(theta[:, nb + 2], 0.3, 1.0)
        _, g = _autograd_grad(ev, theta)
        prop = proposal_from_params(theta, nb, P.table)
        c_ref, d_ref = O.ref_evaluate(P, prop)
        want = -0.5 * fp.stack_grad(d_ref)
        ok = np.abs(g - want) <= GRAD_RTOL * np.abs(want)
        if not np.all(ok):
            # per-band check with the condition-scale criterion of the parity tests
            from test_gpu_parity import check_grad
            ev.run(_torch().as_tensor(theta, device="cuda"), grad=True)
            d_gpu = ev.dchi2.cpu().numpy().reshape(d_ref.shape)
            check_grad(d_gpu, d_ref, P, prop)
        fracs.append(np.mean(ok))
    print("single-source patch: fraction of components within 1e-5 of the reference:", np.mean(fracs))
    P.free()


# ------------------------------------------------------------------ posterior, leapfrog
def _posterior(P, mode="fused"):
    from forcepho_b200.autograd import DevicePosterior, default_bounds
    lo, hi = default_bounds(P.params, P.n_bands)
    return DevicePosterior(P, lo, hi, mode=mode)


def test_lnprob_and_grad_equals_autograd():
    torch = _torch()
    from forcepho_b200 import synth
    P = synth.make_workload("field20", seed=4)
    P.send_to_device()
    post = _posterior(P)
    z = post.inverse_transform(P.params.reshape(-1))
    lnp, g = post.lnprob_and_grad(z)
    zz = z.clone().requires_grad_(True)
    lnp2 = post.lnprob(zz)
    (g2,) = torch.autograd.grad(lnp2, zz)
    # lnprob_and_grad sums lnp in its own fixed order (fpho_bounded_lnp_grad),
    # torch's autograd path in torch's: equal to rounding
    assert abs(float(lnp) - float(lnp2)) <= 1e-14 * abs(float(lnp2))
    np.testing.assert_allclose(g.cpu().numpy(), g2.cpu().numpy(), rtol=1e-13, atol=0)
    P.free()


def test_posterior_matches_fastposterior():
    """DevicePosterior against the host FastPosterior (GPUProposer + host
    BoundedTransform) at the same z."""
    from forcepho_b200 import synth
    from forcepho_b200.model import FastPosterior
    from forcepho_b200.proposal import GPUProposer
    from forcepho_b200.sources import Scene
    from forcepho_b200.autograd import default_bounds
    P = synth.make_workload("field20", seed=4)
    P.send_to_device()
    lo, hi = default_bounds(P.params, P.n_bands)
    post = _posterior(P)
    scene = Scene(P.n_sources, P.n_bands, P.table)
    fp = FastPosterior(GPUProposer(), P, scene=scene, lower=lo, upper=hi)
    z = fp.transform.inverse_transform(P.params.reshape(-1))
    lnp_h, g_h = fp.lnprob_and_grad(z)
    lnp_d, g_d = post.lnprob_and_grad(_torch().as_tensor(z, device="cuda"))
    assert abs(float(lnp_d) - lnp_h) <= 1e-9 * abs(lnp_h)
    np.testing.assert_allclose(g_d.cpu().numpy(), g_h, rtol=1e-6,
                               atol=1e-9 * np.abs(g_h).max())
    P.free()


@pytest.mark.parametrize("use_autograd", [False, True])
def test_leapfrog_graph_equals_eager(use_autograd):
    torch = _torch()
    from forcepho_b200 import synth
    from forcepho_b200.autograd import Leapfrog
    P = synth.make_workload("field20", seed=6)
    P.send_to_device()
    post = _posterior(P)
    z0 = post.inverse_transform(P.params.reshape(-1))
    p0 = torch.as_tensor(np.random.default_rng(1).standard_normal(post.ndim), device="cuda")
    out = []
    for graph in (False, True):
        lf = Leapfrog(post, eps=1e-3, steps_per_graph=5, use_autograd=use_autograd,
                      use_graph=graph)
        lf.set_state(z0, p0)
        lf.run(20)
        torch.cuda.synchronize()
        out.append((lf.z.clone(), lf.p.clone(), float(lf.lnp)))
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
    assert post.ev.error_word() == 0
    P.free()


def test_leapfrog_field20_500_steps():
    """The 20-source patch through the autograd Function, 500 leapfrog steps
    of 1e-3 in the unconstrained (unit-scaled) coordinates, graph-captured.
    The leapfrog's energy error is second order in the step when the gradient
    is the derivative of lnp, so halving the step (1000 steps of 5e-4, same
    trajectory length) must cut it about fourfold; a gradient inconsistent
    with lnp leaves an error that does not shrink with the step."""
    torch = _torch()
    from forcepho_b200 import synth
    from forcepho_b200.autograd import Leapfrog
    P = synth.make_workload("field20", seed=0)
    P.send_to_device()
    post = _posterior(P)
    z0 = post.inverse_transform(P.params.reshape(-1))
    p0 = torch.as_tensor(np.random.default_rng(2).standard_normal(post.ndim), device="cuda")
    dh = []
    for eps, n in ((1e-3, 500), (5e-4, 1000)):
        lf = Leapfrog(post, eps=eps, steps_per_graph=50, use_autograd=True)
        lf.set_state(z0, p0)
        h0, lnp0 = float(lf.hamiltonian()), float(lf.lnp)
        lf.run(n)
        torch.cuda.synchronize()
        h1, lnp1 = float(lf.hamiltonian()), float(lf.lnp)
        print(f"20-source patch, leapfrog eps={eps:g} x {n}: lnp {lnp0:.6f} -> {lnp1:.6f}, "
              f"H {h0:.6f} -> {h1:.6f}, dH {h1 - h0:.6g}")
        assert np.isfinite(h1)
        dh.append(abs(h1 - h0))
    ratio = dh[0] / dh[1]
    print(f"20-source patch, leapfrog: dH ratio for a halved step {ratio:.3f}")
    assert 3.0 < ratio < 5.0
    assert post.ev.error_word() == 0
    P.free()


def test_batch_posterior_matches_single_patches():
    torch = _torch()
    from forcepho_b200 import synth
    from forcepho_b200.autograd import BatchPosterior, default_bounds
    from forcepho_b200.batch import PatchBatch
    patches = synth.make_workload("uneven", seed=9, n_patches=5)
    for p in patches:
        p.send_to_device()
    lows, highs = zip(*[default_bounds(p.params, p.n_bands) for p in patches])
    # the batch switches every patch to its tile shape, so that the single-patch
    # evaluations below sum the same tiles in the same order
    batch = PatchBatch(patches)
    singles = [_posterior(p) for p in patches]
    lnp_s, g_s, zs = 0.0, [], []
    for p, post in zip(patches, singles):
        z = post.inverse_transform(p.params.reshape(-1))
        lnp, g = post.lnprob_and_grad(z)
        lnp_s += float(lnp)
        g_s.append(g.cpu().numpy())
        zs.append(z)
    bp = BatchPosterior(batch, lows, highs)
    lnp_b, g_b = bp.lnprob_and_grad(torch.cat(zs))
    torch.cuda.synchronize()
    assert abs(float(lnp_b) - lnp_s) <= 1e-12 * abs(lnp_s)
    np.testing.assert_allclose(g_b.cpu().numpy(), np.concatenate(g_s), rtol=1e-12, atol=0)
    batch.free()
    for p in patches:
        p.free()
