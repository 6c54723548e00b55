"""Many HMC chains advanced together on the device.

The reference samples one patch with littlemcmc's NUTS, one chain per
process, calling ``lnprob_and_grad`` once per leapfrog step
(forcepho/fitting.py:255-342).  :class:`MultiChainHMC` runs static-length
HMC for many chains at once: every chain is a patch of a
:class:`forcepho_b200.autograd.BatchPosterior` (independent device copies of
one patch, see :func:`chain_posterior`, or different patches), so one batched
launch sequence evaluates every chain's leapfrog step.  One HMC iteration --
momentum draw, ``n_leapfrog`` leapfrog steps, per-chain Metropolis test,
selection of the accepted or the old state, recording of the sample -- is
captured in one CUDA graph and replayed.

Mass matrix.  The reference's NUTS takes the covariance of the
unconstrained coordinates z as its inverse mass matrix (``z_cov``, diagonal
or full, adapted during warm-up; forcepho/fitting.py:255-342, 370-413).
Here the inverse mass of chain k is M_k^-1 = L_k L_k^T, given as a diagonal
(``scale``: L = diag(scale), the per-coordinate standard deviations) or, when
every chain has the same number of coordinates, as one lower-triangular
factor per chain (``chol``).  The leapfrog runs in whitened momenta u = L^T p
with unit kinetic energy: u += eps/2 L^T grad, z += eps L u, which is HMC with
mass M = (L L^T)^-1 in z.  :func:`estimate_mass` turns warm-up samples into
the factors (regularised towards the identity as Stan does).

Step size.  During warm-up the step size adapts inside the captured
iteration by dual averaging (Hoffman & Gelman 2014, the NUTS paper's
Algorithm 5) towards a target mean acceptance probability over the chains;
:meth:`MultiChainHMC.start_adaptation` / :meth:`stop_adaptation` switch it on
and off without re-capturing, and stopping fixes the averaged step size.
"""

import torch

from .autograd import BatchPosterior
from .batch import PatchBatch
from .patches.device_patch import DevicePatch

__all__ = ["MultiChainHMC", "ChainCopy", "chain_posterior", "estimate_mass"]


class ChainCopy:
    """One more device copy of a patch (its own workspace), for one chain."""

    def __init__(self, patch):
        self.n_bands, self.n_sources = patch.n_bands, patch.n_sources
        self.table = getattr(patch, "table", None)
        self.device_patch = DevicePatch(patch, return_residual=False)

    def free(self):
        self.device_patch.free()


def chain_posterior(patch, n_chains, lower, upper, live_cap=128, config=None):
    """A BatchPosterior over `n_chains` device copies of `patch` with the
    same bounds: chain k's parameters are the k-th block of z.  `config`: the
    batched launch configuration (a dict as from
    :func:`forcepho_b200.autotune.choose_batch_config`, or "tune" to have the
    batch autotuner choose it for these copies); None keeps the batch default
    with `live_cap` records per stage."""
    copies = [ChainCopy(patch) for _ in range(n_chains)]
    if isinstance(config, str):
        if config != "tune":
            raise ValueError(f"config must be a dict, 'tune' or None, not {config!r}")
        from .autotune import choose_batch_config
        config = choose_batch_config(copies)
    batch = PatchBatch(copies, live_cap=live_cap, config=config)
    post = BatchPosterior(batch, [lower] * n_chains, [upper] * n_chains)
    post.copies = copies
    return post


def _per_patch(post, v):
    """Sum of a parameter-length vector over each patch's block."""
    return torch.cat([v, v.new_zeros(1)])[post.par_pad].sum(dim=1)


def estimate_mass(samples, n_chains, full=False, pooled=False, shrink=5.0, floor=1e-3):
    """Inverse-mass factors from samples of z (a (n, ndim) tensor, chains
    concatenated along ndim): the per-coordinate standard deviations
    (diagonal) or, with `full`, one Cholesky factor of the covariance per
    chain (every chain must have ndim / n_chains coordinates).  `pooled`
    averages the (co)variances over the chains (chains of one posterior).
    The estimate over N samples is regularised towards `floor` times the
    identity with weight shrink / (N + shrink)."""
    x = samples.to(torch.float64)
    n = x.shape[0]
    w = n / (n + shrink)
    reg = floor * shrink / (n + shrink)
    if not full:
        var = x.var(dim=0, unbiased=True)
        if pooled:
            var = var.view(n_chains, -1).mean(dim=0).repeat(n_chains)
        return (w * var + reg).sqrt()
    d = x.shape[1] // n_chains
    xc = x.view(n, n_chains, d)
    xc = xc - xc.mean(dim=0, keepdim=True)
    cov = torch.einsum("nki,nkj->kij", xc, xc) / max(n - 1, 1)
    if pooled:
        cov = cov.mean(dim=0, keepdim=True).expand(n_chains, d, d)
    eye = torch.eye(d, dtype=torch.float64, device=x.device)
    return torch.linalg.cholesky(w * cov + reg * eye)


class MultiChainHMC:
    """Static-length HMC with a Metropolis test per chain.

    posterior: a BatchPosterior (``lnprob_and_grad``, ``lnp_per_patch``,
    ``par_patch``, ``par_pad``, ``n_patches``, ``ndim``); each patch is one
    chain.  ``n_samples`` > 0 keeps the last that many states in
    ``samples`` (a ring buffer on the device).  Each iteration draws each
    chain's step size uniformly in eps * (1 +- jitter).  The inverse mass
    matrix is the identity until :meth:`set_mass` (``full``: one dense
    factor per chain, which needs chains of equal size).
    """

    def __init__(self, posterior, eps, n_leapfrog, n_samples=0, seed=0, jitter=0.2,
                 full=False, device="cuda"):
        self.post = posterior
        self.device = torch.device(device)
        dev = self.device
        # the step size lives on the device, so a captured iteration reads the
        # current value (set_eps between replays tunes it)
        self.eps_t = torch.full((), float(eps), dtype=torch.float64, device=dev)
        self.jitter = float(jitter)
        self.L = int(n_leapfrog)
        n, k = posterior.ndim, posterior.n_patches
        f64 = dict(dtype=torch.float64, device=dev)
        self.z, self.g = torch.zeros(n, **f64), torch.zeros(n, **f64)
        self.lnp = torch.zeros(k, **f64)
        self.n_accept = torch.zeros(k, dtype=torch.int64, device=dev)
        self.n_samples = int(n_samples)
        self.samples = torch.zeros((max(self.n_samples, 1), n), **f64)
        self.slot = torch.zeros(1, dtype=torch.int64, device=dev)
        # inverse-mass factors, read by the captured graph: set_mass copies into them
        self.scale = torch.ones(n, **f64)
        self.full = bool(full)
        self.chol = None
        if self.full:
            if n % k:
                raise ValueError("a full mass matrix needs chains of equal size")
            d = n // k
            self.chol = torch.eye(d, **f64).repeat(k, 1, 1)
        # dual-averaging state (device scalars, so the captured graph adapts)
        self.da_on = torch.zeros((), **f64)        # 1 while adapting
        self.da_m = torch.zeros((), **f64)         # adaptation iterations
        self.da_hbar = torch.zeros((), **f64)
        self.da_mu = torch.zeros((), **f64)
        self.da_logbar = torch.zeros((), **f64)
        self.da_target = torch.full((), 0.8, **f64)
        self.mean_accept_prob = torch.zeros((), **f64)
        self.graph = None
        if dev.type == "cuda":
            torch.cuda.manual_seed(seed)
        else:
            torch.manual_seed(seed)

    # dual-averaging constants (gamma, t0, kappa of Hoffman & Gelman 2014)
    DA_GAMMA, DA_T0, DA_KAPPA = 0.05, 10.0, 0.75

    def start_adaptation(self, target_accept=0.8):
        """Adapt the step size from the next iteration on, starting from the
        current one (mu = log(10 eps))."""
        self.da_on.fill_(1.0)
        self.da_m.zero_()
        self.da_hbar.zero_()
        self.da_mu.copy_(torch.log(10.0 * self.eps_t))
        self.da_logbar.copy_(torch.log(self.eps_t))
        self.da_target.fill_(float(target_accept))

    def stop_adaptation(self):
        """Stop adapting and keep the averaged step size."""
        self.da_on.zero_()
        self.eps_t.copy_(torch.exp(self.da_logbar))

    def _adapt(self, accept_prob):
        """One dual-averaging update from this iteration's mean acceptance
        probability (no effect while da_on is 0)."""
        f = self.da_on
        m = self.da_m + f
        eta = 1.0 / (m + self.DA_T0)
        self.da_hbar.copy_((1.0 - f * eta) * self.da_hbar + f * eta * (self.da_target - accept_prob))
        log_eps = self.da_mu - torch.sqrt(m) / self.DA_GAMMA * self.da_hbar
        w = torch.pow(torch.clamp(m, min=1.0), -self.DA_KAPPA)
        self.da_logbar.copy_(f * (w * log_eps + (1.0 - w) * self.da_logbar) +
                             (1.0 - f) * self.da_logbar)
        self.eps_t.copy_(f * torch.exp(log_eps) + (1.0 - f) * self.eps_t)
        self.da_m.copy_(m)

    def set_mass(self, scale=None, chol=None):
        """Inverse mass matrix: per-coordinate standard deviations `scale`
        (ndim,) or, for a sampler made with ``full``, Cholesky factors `chol`
        (n_chains, d, d) or (d, d) for every chain.  Takes effect in the next
        iteration (graph replays included)."""
        if scale is not None:
            self.scale.copy_(torch.as_tensor(scale, dtype=torch.float64).reshape(-1))
        if chol is not None:
            if self.chol is None:
                raise ValueError("the sampler was made without a full mass matrix")
            c = torch.as_tensor(chol, dtype=torch.float64, device=self.device)
            self.chol.copy_(c.expand_as(self.chol))

    def _to_z(self, u):
        """L u per chain: a whitened displacement in z."""
        if self.chol is None:
            return self.scale * u
        k, d = self.chol.shape[0], self.chol.shape[1]
        return torch.bmm(self.chol, u.view(k, d, 1)).view(-1)

    def _to_u(self, g):
        """L^T g per chain: a z-gradient in whitened coordinates."""
        if self.chol is None:
            return self.scale * g
        k, d = self.chol.shape[0], self.chol.shape[1]
        return torch.bmm(self.chol.transpose(1, 2), g.view(k, d, 1)).view(-1)

    @property
    def eps(self):
        return float(self.eps_t)

    def set_eps(self, eps):
        """New base step size for the following iterations (graph included)."""
        self.eps_t.fill_(float(eps))

    def set_state(self, z0):
        self.z.copy_(torch.as_tensor(z0, dtype=torch.float64))
        _, g = self.post.lnprob_and_grad(self.z)
        self.g.copy_(g)
        self.lnp.copy_(self.post.lnp_per_patch(self.z))

    def _iteration(self):
        post = self.post
        # a step size per chain, drawn uniformly within +-jitter of eps, so that
        # a fixed trajectory length cannot lock onto a period of the dynamics
        u = torch.rand(self.lnp.shape, dtype=torch.float64, device=self.device)
        eps = (self.eps_t * (1.0 + self.jitter * (2.0 * u - 1.0)))[post.par_patch]
        h = 0.5 * eps
        p = torch.randn(self.z.shape, dtype=torch.float64, device=self.device)  # whitened momenta
        kin0 = _per_patch(post, p * p) * 0.5
        z, g = self.z.clone(), self.g.clone()
        if self.chol is None:
            # diagonal mass: kick p += (h scale) g, drift z += (eps scale) p,
            # one launch each
            hs, es = h * self.scale, eps * self.scale
            for _ in range(self.L):
                p.addcmul_(hs, g)
                z.addcmul_(es, p)
                _, g = post.lnprob_and_grad(z)
                p.addcmul_(hs, g)
        else:
            gu = self._to_u(g)
            for _ in range(self.L):
                p = p + h * gu
                z = z + eps * self._to_z(p)
                _, g = post.lnprob_and_grad(z)
                gu = self._to_u(g)
                p = p + h * gu
        lnp1 = post.lnp_per_patch(z)
        kin1 = _per_patch(post, p * p) * 0.5
        log_ratio = (lnp1 - kin1) - (self.lnp - kin0)
        ok = torch.isfinite(log_ratio)
        prob = torch.where(ok, torch.exp(torch.clamp(torch.nan_to_num(log_ratio), max=0.0)),
                           torch.zeros_like(log_ratio))
        self.mean_accept_prob.copy_(prob.mean())
        self._adapt(self.mean_accept_prob)
        u = torch.rand(self.lnp.shape, dtype=torch.float64, device=self.device)
        acc = (torch.log(u) < log_ratio) & torch.isfinite(lnp1)
        accp = acc[post.par_patch]
        self.z.copy_(torch.where(accp, z, self.z))
        self.g.copy_(torch.where(accp, g, self.g))
        self.lnp.copy_(torch.where(acc, lnp1, self.lnp))
        self.n_accept.add_(acc.to(torch.int64))
        if self.n_samples:
            self.samples.index_copy_(0, self.slot % self.n_samples, self.z.unsqueeze(0))
            self.slot.add_(1)

    def _capture(self):
        state = (self.z, self.g, self.lnp, self.n_accept, self.slot)
        saved = [t.clone() for t in state]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self._iteration()  # warm-up outside capture
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        for t, v in zip(state, saved):
            t.copy_(v)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._iteration()

    def run(self, n_iter, use_graph=True):
        """Advance every chain by `n_iter` HMC iterations (enqueued on the
        current stream, not synchronized; one CUDA graph replay per iteration
        on a GPU, plain eager iterations on the CPU)."""
        if not use_graph or self.device.type != "cuda":
            for _ in range(n_iter):
                self._iteration()
            return
        if self.graph is None:
            self._capture()
        for _ in range(n_iter):
            self.graph.replay()

    def acceptance(self, n_iter):
        """Fraction of accepted iterations per chain."""
        return (self.n_accept.to(torch.float64) / max(n_iter, 1)).cpu().numpy()
