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
"""

import torch

from .autograd import BatchPosterior
from .batch import PatchBatch
from .patches.device_patch import DevicePatch

__all__ = ["MultiChainHMC", "ChainCopy", "chain_posterior"]


class ChainCopy:
    """One more device copy of a patch (its own workspace), for one chain."""

    def __init__(self, patch):
        self.n_bands, self.n_sources = patch.n_bands, patch.n_sources
        self.table = getattr(patch, "table", None)
        self.device_patch = DevicePatch(patch, return_residual=False)

    def free(self):
        self.device_patch.free()


def chain_posterior(patch, n_chains, lower, upper, live_cap=128):
    """A BatchPosterior over `n_chains` device copies of `patch` with the
    same bounds: chain k's parameters are the k-th block of z."""
    copies = [ChainCopy(patch) for _ in range(n_chains)]
    batch = PatchBatch(copies, live_cap=live_cap)
    post = BatchPosterior(batch, [lower] * n_chains, [upper] * n_chains)
    post.copies = copies
    return post


def _per_patch(post, v):
    """Sum of a parameter-length vector over each patch's block."""
    return torch.cat([v, v.new_zeros(1)])[post.par_pad].sum(dim=1)


class MultiChainHMC:
    """Static-length HMC (unit mass) with a Metropolis test per chain.

    posterior: a BatchPosterior (``lnprob_and_grad``, ``lnp_per_patch``,
    ``par_patch``, ``par_pad``, ``n_patches``, ``ndim``); each patch is one
    chain.  ``n_samples`` > 0 keeps the last that many states in
    ``samples`` (a ring buffer on the device).  Each iteration draws each
    chain's step size uniformly in eps * (1 +- jitter).
    """

    def __init__(self, posterior, eps, n_leapfrog, n_samples=0, seed=0, jitter=0.2):
        self.post = posterior
        # the step size lives on the device, so a captured iteration reads the
        # current value (set_eps between replays tunes it)
        self.eps_t = torch.full((), float(eps), dtype=torch.float64, device="cuda")
        self.jitter = float(jitter)
        self.L = int(n_leapfrog)
        n, k = posterior.ndim, posterior.n_patches
        f64 = dict(dtype=torch.float64, device="cuda")
        self.z, self.g = torch.zeros(n, **f64), torch.zeros(n, **f64)
        self.lnp = torch.zeros(k, **f64)
        self.n_accept = torch.zeros(k, dtype=torch.int64, device="cuda")
        self.n_samples = int(n_samples)
        self.samples = torch.zeros((max(self.n_samples, 1), n), **f64)
        self.slot = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.graph = None
        torch.cuda.manual_seed(seed)

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
        u = torch.rand(self.lnp.shape, dtype=torch.float64, device="cuda")
        eps = (self.eps_t * (1.0 + self.jitter * (2.0 * u - 1.0)))[post.par_patch]
        h = 0.5 * eps
        p = torch.randn(self.z.shape, dtype=torch.float64, device="cuda")
        kin0 = _per_patch(post, p * p) * 0.5
        z, g = self.z.clone(), self.g.clone()
        for _ in range(self.L):
            p = p + h * g
            z = z + eps * p
            _, g = post.lnprob_and_grad(z)
            p = p + h * g
        lnp1 = post.lnp_per_patch(z)
        kin1 = _per_patch(post, p * p) * 0.5
        log_ratio = (lnp1 - kin1) - (self.lnp - kin0)
        u = torch.rand(self.lnp.shape, dtype=torch.float64, device="cuda")
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
        current stream, not synchronized)."""
        if not use_graph:
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
