"""CPU: the many-chain HMC sampler's host-independent logic on analytic
targets, with CPU tensors (the CUDA-graph replay is a GPU path; the
iteration itself is the same code):

  * estimate_mass: per-coordinate standard deviations and per-chain
    Cholesky factors of sample covariances, pooled over chains, regularised
    towards the identity;
  * dual averaging of the step size inside the iteration: the chains' mean
    acceptance probability ends near the target;
  * run_hmc with a diagonal or a dense adapted mass matrix recovers the
    target's (co)variances, and the production samples follow the target.
"""
import numpy as np
import pytest
import torch

from forcepho_b200.fitting import run_hmc
from forcepho_b200.sampling import MultiChainHMC, estimate_mass


class Target:
    """K chains of d coordinates: lnp = -1/2 (z-mu)^T C^-1 (z-mu) per chain,
    one covariance C for every chain, identity transform."""
    device = "cpu"

    def __init__(self, k, C, seed=0):
        rng = np.random.default_rng(seed)
        d = C.shape[0]
        self.k, self.d = k, d
        self.n_patches, self.ndim = k, k * d
        self.C = C
        self.Ci = torch.as_tensor(np.linalg.inv(C))
        self.mu = torch.as_tensor(rng.normal(size=k * d))
        self.par_patch = torch.as_tensor(np.repeat(np.arange(k), d))
        self.par_pad = torch.as_tensor(np.arange(k * d).reshape(k, d))
        self.copies = [None] * k  # chains of one posterior: estimates pool

    def _r(self, z):
        x = (z - self.mu).view(self.k, self.d)
        return x, x @ self.Ci

    def lnprob_and_grad(self, z):
        x, y = self._r(z)
        return -0.5 * (x * y).sum(), -y.reshape(-1)

    def lnp_per_patch(self, z):
        x, y = self._r(z)
        return -0.5 * (x * y).sum(dim=1)

    def transform(self, z):
        return z

    def inverse_transform(self, q):
        return torch.as_tensor(q, dtype=torch.float64)


def _aniso(d=5, seed=1):
    rng = np.random.default_rng(seed)
    return np.diag(np.exp(rng.uniform(np.log(0.02), np.log(5.0), size=d)) ** 2)


def test_estimate_mass_diag_full_pooled():
    rng = np.random.default_rng(0)
    k, d, n = 8, 3, 4000
    A = np.array([[1.0, 0.0, 0.0], [0.8, 0.6, 0.0], [0.1, 0.2, 0.3]])
    C = A @ A.T
    x = torch.as_tensor(rng.standard_normal((n, k, d)) @ A.T).reshape(n, k * d)
    s = estimate_mass(x, k, pooled=True)
    np.testing.assert_allclose(s.numpy().reshape(k, d)[0] ** 2, np.diag(C), rtol=0.06)
    assert torch.equal(s.view(k, d)[0], s.view(k, d)[-1])       # pooled: every chain the same
    L = estimate_mass(x, k, full=True, pooled=True)
    assert L.shape == (k, d, d) and torch.allclose(L, torch.tril(L))
    np.testing.assert_allclose((L[0] @ L[0].T).numpy(), C, atol=0.06)
    # per chain, and the regularisation towards floor * identity at few samples
    Lk = estimate_mass(x[:5], k, full=True)
    assert Lk.shape == (k, d, d) and torch.all(torch.isfinite(Lk))
    s1 = estimate_mass(x[:2] * 0.0, k, floor=1e-3)               # no spread: the floor
    np.testing.assert_allclose(s1.numpy() ** 2, 1e-3 * 5 / 7, rtol=1e-12)


def test_dual_averaging_reaches_target_acceptance():
    T = Target(32, np.eye(4))
    hmc = MultiChainHMC(T, eps=1e-3, n_leapfrog=8, seed=2, device="cpu")
    hmc.set_state(T.mu.clone())
    hmc.start_adaptation(0.8)
    hmc.run(300)
    hmc.stop_adaptation()
    assert 0.2 < hmc.eps < 2.0        # grew from 1e-3 towards the unit target's scale
    hmc.n_accept.zero_()
    hmc.run(200)
    acc = hmc.acceptance(200).mean()
    assert 0.65 < acc < 0.95, acc


@pytest.mark.parametrize("full", [False, True])
def test_run_hmc_adapts_mass(full):
    if full:
        s = np.array([0.05, 0.5, 2.0])
        r = np.array([[1.0, 0.95, 0.3], [0.95, 1.0, 0.5], [0.3, 0.5, 1.0]])
        C = s[:, None] * r * s[None, :]
    else:
        C = _aniso()
    T = Target(32, C, seed=3)
    res, hmc = run_hmc(T, T.mu.numpy(), n_draws=300, warmup=[100, 100, 100], n_leapfrog=8,
                       step_size=0.01, adapt=True, full=full, random_seed=4)
    sd = np.sqrt(np.diag(C))
    if full:
        L = hmc.chol[0]
        err = np.abs((L @ L.T).numpy() - C) / (sd[:, None] * sd[None, :])
        assert err.max() < 0.12, err.max()
    else:
        ratio = hmc.scale.numpy().reshape(T.k, T.d)[0] ** 2 / np.diag(C)
        assert np.all((ratio > 0.8) & (ratio < 1.25)), ratio
    chain = res.chain                                    # (chains, draws, d)
    v = chain.transpose(1, 0, 2).reshape(300, -1).var(axis=0).reshape(T.k, T.d).mean(axis=0)
    np.testing.assert_allclose(v / np.diag(C), 1.0, atol=0.2)
    assert res.accept.mean() > 0.5


def test_param_maps_group_in_order():
    """The CSR maps of the fused gradient keep each parameter's entries in the
    order given (band order for the shape parameters)."""
    from forcepho_b200.autograd import _param_maps
    dst = [2, 0, 2, 1, 2, 0]
    src = [10, 11, 12, 13, 14, 15]
    off, idx = _param_maps(4, dst, src)
    assert off.tolist() == [0, 2, 3, 6, 6]
    assert idx.tolist() == [11, 15, 13, 10, 12, 14]


def test_fused_posterior_refuses_bad_z():
    """The fused launches read z as ndim float64 values on the GPU: a z of
    another type, device or length is refused before any launch."""
    import torch
    from forcepho_b200.autograd import _device_z
    for bad in (np.zeros(3), torch.zeros(3), torch.zeros(3, dtype=torch.float32)):
        with pytest.raises(TypeError):
            _device_z(bad, 3)
