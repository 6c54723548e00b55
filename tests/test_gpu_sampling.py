"""GPU: many HMC chains in one batched launch sequence (forcepho_b200.sampling).

  * the sampler's mechanics on an analytic target (independent Gaussians per
    chain, no patch): after burn-in, the sample means are within 0.05 sigma
    of the truth on average (0.2 at worst) and the variances within 10% on
    average (0.7..1.4 at worst);
  * chain copies of one patch: each chain's lnp and gradient equal the
    single-patch device posterior's at the same z (1e-12 relative) and the
    per-chain lnp sum to the total;
  * a short run on the single-source patch: every chain finite, moved, and
    accepting more than half of its proposals; the batched kernels' error
    word stays 0.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class GaussianTarget:
    """lnp = -0.5 sum ((z - mu) / sigma)^2 per chain; K chains of d coordinates."""

    def __init__(self, k, d, seed=0):
        import torch
        rng = np.random.default_rng(seed)
        self.n_patches, self.ndim = k, k * d
        self.mu = torch.as_tensor(rng.normal(size=k * d), device="cuda")
        self.sig = torch.as_tensor(rng.uniform(0.5, 2.0, size=k * d), device="cuda")
        self.par_patch = torch.as_tensor(np.repeat(np.arange(k), d), device="cuda")
        self.par_pad = torch.as_tensor(np.arange(k * d).reshape(k, d), device="cuda")
        self._last = None

    def lnprob_and_grad(self, z):
        r = (z - self.mu) / self.sig
        self._last = -0.5 * r * r
        return self._last.sum(), -r / self.sig

    def lnp_per_patch(self, z):
        r = (z - self.mu) / self.sig
        return (-0.5 * r * r)[self.par_pad].sum(dim=1)


def test_hmc_on_gaussian_target():
    import torch
    from forcepho_b200.sampling import MultiChainHMC
    T = GaussianTarget(64, 3)
    n_iter, burn = 1500, 100
    hmc = MultiChainHMC(T, eps=0.25, n_leapfrog=8, n_samples=n_iter - burn, seed=1)
    hmc.set_state(torch.zeros(T.ndim, dtype=torch.float64, device="cuda"))
    hmc.run(burn)
    hmc.run(n_iter - burn)
    torch.cuda.synchronize()
    smp = hmc.samples.cpu().numpy()
    mu, sig = T.mu.cpu().numpy(), T.sig.cpu().numpy()
    m = smp.mean(axis=0)
    v = smp.var(axis=0)
    acc = hmc.acceptance(n_iter)
    print(f"gaussian target: acceptance {acc.mean():.3f}, max |mean - mu| / sigma "
          f"{np.max(np.abs(m - mu) / sig):.3f}, variance ratio "
          f"{np.min(v / sig**2):.3f}..{np.max(v / sig**2):.3f}")
    assert np.mean(np.abs(m - mu) / sig) < 0.05
    assert abs(np.mean(v / sig**2) - 1.0) < 0.1
    assert np.max(np.abs(m - mu) / sig) < 0.2
    assert 0.7 < np.min(v / sig**2) and np.max(v / sig**2) < 1.4
    assert acc.min() > 0.5


def _chains(P, k):
    from forcepho_b200.autograd import default_bounds
    from forcepho_b200.sampling import chain_posterior
    lo, hi = default_bounds(P.params, P.n_bands)
    return chain_posterior(P, k, lo, hi), lo, hi


def test_chain_copies_match_single_patch():
    import torch
    from forcepho_b200 import synth
    from forcepho_b200.autograd import DevicePosterior
    P = synth.make_workload("field20", seed=3)
    post, lo, hi = _chains(P, 3)
    P.send_to_device()
    # the batch evaluates 64x8 tiles with 128-record stages: same for the single patch
    from forcepho_b200 import _lib
    v = [i for i, (nt, k) in enumerate(_lib.variants()) if (nt, k) == (64, 8)][0]
    P.device_patch.set_config(v, 128)
    single = DevicePosterior(P, lo, hi)
    rng = np.random.default_rng(0)
    z0 = single.inverse_transform(P.params.reshape(-1))
    zs = [z0 + torch.as_tensor(0.01 * rng.standard_normal(z0.shape), device="cuda")
          for _ in range(3)]
    lnp, g = post.lnprob_and_grad(torch.cat(zs))
    per = post.lnp_per_patch(torch.cat(zs))
    torch.cuda.synchronize()
    assert abs(float(per.sum()) - float(lnp)) <= 1e-12 * abs(float(lnp))
    n = z0.numel()
    for k, z in enumerate(zs):
        l1, g1 = single.lnprob_and_grad(z)
        assert abs(float(per[k]) - float(l1)) <= 1e-12 * abs(float(l1))
        np.testing.assert_allclose(g[k * n:(k + 1) * n].cpu().numpy(), g1.cpu().numpy(),
                                   rtol=1e-12, atol=0)
    for c in post.copies:
        c.free()
    P.free()


def test_many_chains_on_single_source_patch():
    import torch
    from forcepho_b200 import synth
    from forcepho_b200.sampling import MultiChainHMC
    P = synth.make_workload("single", seed=2)
    k = 32
    post, lo, hi = _chains(P, k)
    z0 = post.inverse_transform(np.tile(P.params.reshape(-1), k))
    hmc = MultiChainHMC(post, eps=5e-3, n_leapfrog=10, seed=3)
    hmc.set_state(z0)
    hmc.run(100)
    torch.cuda.synchronize()
    acc = hmc.acceptance(100)
    z = hmc.z.cpu().numpy().reshape(k, -1)
    print(f"single-source patch, {k} chains: acceptance {acc.mean():.3f} "
          f"(min {acc.min():.3f}), lnp {hmc.lnp.cpu().numpy().mean():.3f}")
    assert np.all(np.isfinite(z)) and np.all(np.isfinite(hmc.lnp.cpu().numpy()))
    assert np.all(np.any(z != z0.cpu().numpy().reshape(k, -1), axis=1))
    assert acc.mean() > 0.5
    assert post.batch.error_word() == 0
    post.batch.free()
    for c in post.copies:
        c.free()


def test_run_hmc_and_run_opt_call_shapes():
    """fitting.run_hmc / run_opt keep the call shape and result fields of the
    reference's run_lmc / run_opt (fitting.py:255-342, 415-454): chains in the
    constrained space inside the bounds, call counts, a tuned step size that
    a captured graph picks up, and BFGS raising the posterior."""
    from forcepho_b200 import synth
    from forcepho_b200.autograd import DevicePosterior, default_bounds
    from forcepho_b200.fitting import run_hmc, run_opt
    from forcepho_b200.model import FastPosterior
    from forcepho_b200.proposal import GPUProposer
    from forcepho_b200.sources import Scene
    P = synth.make_workload("single", seed=4)
    P.send_to_device()
    lo, hi = default_bounds(P.params, P.n_bands)
    post = DevicePosterior(P, lo, hi)
    q0 = P.params.reshape(-1)
    res, hmc = run_hmc(post, q0, n_draws=40, warmup=[30, 30], n_chains=4, n_leapfrog=8,
                       step_size=0.05)
    assert res.chain.shape == (4, 40, q0.size)
    assert np.all(res.chain >= lo) and np.all(res.chain <= hi)
    assert res.n_call == 4 * (60 + 40) * 8 and res.wall_time > 0
    assert np.all(np.isfinite(res.chain)) and np.all(res.chain.std(axis=1) > 0)
    assert 0.3 < res.accept.mean() <= 1.0 and res.step_size != 0.05
    one, _ = run_hmc(post, q0, n_draws=10, warmup=[10], n_chains=1, n_leapfrog=5)
    assert one.chain.shape == (10, q0.size)
    fp = FastPosterior(GPUProposer(), P, scene=Scene(P.n_sources, P.n_bands, P.table),
                       lower=lo, upper=hi)
    start = 0.5 * (lo + hi) + 0.1 * (q0 - 0.5 * (lo + hi))
    r, sci = run_opt(fp, start, maxiter=50)
    assert r.chain.shape == (1, q0.size) and np.isfinite(r.lnp)
    lnp_start = fp.lnprob(fp.transform.inverse_transform(start))
    lnp_end = fp.lnprob(fp.transform.inverse_transform(r.chain[0]))
    assert lnp_end > lnp_start
    P.free()


class AnisoTarget(GaussianTarget):
    """Independent Gaussians with standard deviations spread log-uniformly
    over [0.02, 5] (a 250x range), identity transform."""

    def __init__(self, k, d, seed=0):
        import torch
        super().__init__(k, d, seed)
        rng = np.random.default_rng(seed + 1)
        sd = np.exp(rng.uniform(np.log(0.02), np.log(5.0), size=d))
        self.sig = torch.as_tensor(np.tile(sd, k), device="cuda")

    def transform(self, z):
        return z

    def inverse_transform(self, q):
        import torch
        return torch.as_tensor(q, dtype=torch.float64, device="cuda")


class CorrTarget(AnisoTarget):
    """One correlated 3-D Gaussian per chain: lnp = -1/2 (z-mu)^T C^-1 (z-mu)
    with correlations up to 0.95 and scales 0.05..2."""

    def __init__(self, k, seed=0):
        import torch
        super().__init__(k, 3, seed)
        s = np.array([0.05, 0.5, 2.0])
        r = np.array([[1.0, 0.95, 0.3], [0.95, 1.0, 0.5], [0.3, 0.5, 1.0]])
        self.C = s[:, None] * r * s[None, :]
        self.Ci = torch.as_tensor(np.linalg.inv(self.C), device="cuda")
        self.k = k

    def _r(self, z):
        x = (z - self.mu).view(self.k, 3)
        return x, x @ self.Ci

    def lnprob_and_grad(self, z):
        x, y = self._r(z)
        return -0.5 * (x * y).sum(), -y.reshape(-1)

    def lnp_per_patch(self, z):
        x, y = self._r(z)
        return -0.5 * (x * y).sum(dim=1)


def test_diagonal_mass_adaptation():
    """run_hmc with adapt: the inverse mass recovers the target's variances
    within 10% on average (each within 0.7..1.4), the production samples'
    variances follow, and at one fixed step size the adapted mass accepts far
    more often than the identity."""
    import torch
    from forcepho_b200.fitting import run_hmc
    from forcepho_b200.sampling import MultiChainHMC
    T = AnisoTarget(64, 6, seed=3)
    T.copies = [None] * 64          # chains of one posterior: pool the estimates
    q0 = T.mu.cpu().numpy()
    res, hmc = run_hmc(T, q0, n_draws=400, warmup=[100, 100, 100], n_leapfrog=10,
                       step_size=0.01, adapt=True, random_seed=5)
    sig2 = (T.sig ** 2).cpu().numpy()
    ratio = (hmc.scale ** 2).cpu().numpy() / sig2
    v = res.chain.reshape(-1, 6 * 64).var(axis=0) if res.chain.ndim == 2 else \
        res.chain.transpose(1, 0, 2).reshape(400, -1).var(axis=0)
    print(f"diagonal adaptation: mass/variance ratio {ratio.mean():.3f} "
          f"({ratio.min():.3f}..{ratio.max():.3f}); sample variance ratio "
          f"{np.mean(v / sig2):.3f}; step size {res.step_size:.3f}; acceptance "
          f"{res.accept.mean():.3f}")
    assert abs(ratio.mean() - 1.0) < 0.1 and 0.7 < ratio.min() and ratio.max() < 1.4
    assert abs(np.mean(v / sig2) - 1.0) < 0.15
    acc = {}
    for name, scale in (("identity", None), ("adapted", hmc.scale)):
        h = MultiChainHMC(T, eps=0.3, n_leapfrog=10, seed=7)
        if scale is not None:
            h.set_mass(scale=scale)
        h.set_state(T.mu.clone())
        h.run(50)
        acc[name] = float(h.acceptance(50).mean())
    print("acceptance at eps 0.3:", acc)
    assert acc["adapted"] > acc["identity"] + 0.3


def test_full_mass_adaptation():
    """run_hmc with full and adapt on correlated 3-D Gaussians: the
    inverse-mass factor L recovers the covariance (L L^T within 10% of C,
    relative to its diagonal scales)."""
    import torch
    from forcepho_b200.fitting import run_hmc
    T = CorrTarget(64, seed=4)
    T.copies = [None] * 64
    res, hmc = run_hmc(T, T.mu.cpu().numpy(), n_draws=300, warmup=[100, 100, 100],
                       n_leapfrog=10, step_size=0.01, adapt=True, full=True, random_seed=9)
    L = hmc.chol[0]
    M = (L @ L.T).cpu().numpy()
    s = np.sqrt(np.diag(T.C))
    err = np.abs(M - T.C) / (s[:, None] * s[None, :])
    print(f"full adaptation: max |LL^T - C| / (s_i s_j) {err.max():.3f}; step size "
          f"{res.step_size:.3f}; acceptance {res.accept.mean():.3f}")
    assert err.max() < 0.1
    assert res.accept.mean() > 0.5
