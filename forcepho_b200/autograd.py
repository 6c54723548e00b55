"""The differentiable form of the proposal evaluation.

:class:`LnLike` is a ``torch.autograd.Function``: forward maps source
parameters theta (float64, Scene order ``[flux_1..flux_B, ra, dec, q, pa,
sersic, rhalf]`` per source) to ``lnlike = -chi2 / 2``; backward returns
``d lnlike / d theta`` from the hand-written adjoint of the tile kernel (the
residual pushed through the image-Gaussian, on-sky-Gaussian and parameter
Jacobians, including d(amplitude)/d(sersic) and d(amplitude)/d(rh) from the
amplitude splines).  Two modes:

  ``fused``      forward runs the residual and gradient passes together and
                 backward only stacks the per-band gradient (one launch
                 sequence per lnlike-and-gradient);
  ``recompute``  forward runs the chi2-only kernel (no gradient pass) and
                 backward re-runs the evaluation with its gradient pass,
                 rebuilding the image Gaussians per tile.

Neither mode stores per-pixel intermediates.  :class:`DevicePosterior` is the
device-resident counterpart of ``FastPosterior`` with a ``BoundedTransform``
(forcepho/model.py:260-405, 596-637): ``lnp = lnlike + sum log|dq/dz|``.
:class:`Leapfrog` integrates Hamiltonian dynamics with unit mass on it and
captures its steps in a CUDA graph (the leapfrog of the reference's NUTS
sampler, forcepho/fitting.py:255-342, calls ``lnprob_and_grad`` once per
step).  :class:`BatchPosterior` does the same for many patches through the
persistent batched kernel.
"""

import numpy as np
import torch

from . import _lib
from .device_proposal import DeviceSersicTable, SOURCE_BYTES
from .kernel_limits import NPARAMS

__all__ = ["PatchEvaluator", "LnLike", "DevicePosterior", "BatchPosterior", "Leapfrog",
           "default_bounds", "stack_grad"]


def _stream():
    return torch.cuda.current_stream().cuda_stream


def stack_grad(dchi2, n_bands, n_sources):
    """(n_bands, n_sources, 7) float32 -> (n_sources, n_bands + 6) float64:
    per-band flux derivatives and shape derivatives summed over bands, as
    FastPosterior.stack_grad (forcepho/model.py:387-405)."""
    d = dchi2.view(n_bands, n_sources, NPARAMS).to(torch.float64)
    return torch.cat([d[:, :, 0].t(), d[:, :, 1:].sum(0)], dim=1)


class PatchEvaluator:
    """Device buffers and launches evaluating one patch at device parameters."""

    def __init__(self, patch, table=None, mode="fused"):
        if mode not in ("fused", "recompute"):
            raise ValueError("mode must be 'fused' or 'recompute'")
        if patch.device_patch is None:
            patch.send_to_device()
        self.patch = patch
        self.handle = patch.device_patch.handle
        self.mode = mode
        self.n_bands, self.n_sources = int(patch.n_bands), int(patch.n_sources)
        self.table = table if isinstance(table, DeviceSersicTable) else \
            DeviceSersicTable(table or getattr(patch, "table", None))
        self.prop = self.table.empty_proposal(self.n_sources)
        self.chi2 = torch.zeros(self.n_bands, dtype=torch.float64, device="cuda")
        self.dchi2 = torch.zeros(self.n_bands * self.n_sources * NPARAMS, dtype=torch.float32,
                                 device="cuda")
        self.generation = 0

    @property
    def n_params(self):
        return self.n_sources * (self.n_bands + 6)

    def run(self, theta, grad=True):
        """Build the proposal from theta and enqueue one evaluation."""
        self.table.build_proposal(theta.reshape(self.n_sources, self.n_bands + 6),
                                  self.n_bands, out=self.prop)
        flags = 0 if grad else _lib.FPHO_CHI2_ONLY
        _lib.call("fpho_evaluate_proposal", self.handle, self.prop.data_ptr(), self.n_sources,
                  self.chi2.data_ptr(), self.dchi2.data_ptr() if grad else None,
                  NPARAMS * self.n_sources, flags, _stream())
        self.generation += 1

    def evaluate(self, grad=True):
        """Enqueue one evaluation of the proposal already in ``self.prop``."""
        flags = 0 if grad else _lib.FPHO_CHI2_ONLY
        _lib.call("fpho_evaluate_proposal", self.handle, self.prop.data_ptr(), self.n_sources,
                  self.chi2.data_ptr(), self.dchi2.data_ptr() if grad else None,
                  NPARAMS * self.n_sources, flags, _stream())
        self.generation += 1

    def stacked(self):
        """d chi2 / d theta of the last gradient run, (n_sources, n_bands + 6)."""
        return stack_grad(self.dchi2, self.n_bands, self.n_sources)

    def error_word(self):
        import ctypes
        w = ctypes.c_int()
        _lib.call("fpho_patch_error_word", self.handle, ctypes.byref(w))
        return w.value


class LnLike(torch.autograd.Function):
    """lnlike(theta) = -sum_b chi2_b / 2 with the hand-written adjoint."""

    @staticmethod
    def forward(ctx, theta, ev):
        fused = ev.mode == "fused"
        ev.run(theta, grad=fused)
        ctx.ev, ctx.fused, ctx.gen = ev, fused, ev.generation
        ctx.save_for_backward(theta)
        return ev.chi2.sum() * -0.5

    @staticmethod
    def backward(ctx, g):
        ev = ctx.ev
        if not ctx.fused or ev.generation != ctx.gen:
            (theta,) = ctx.saved_tensors
            ev.run(theta, grad=True)
        return (ev.stacked() * (g * -0.5)).reshape(ctx.saved_tensors[0].shape), None


def lnlike(theta, ev):
    return LnLike.apply(theta, ev)


def default_bounds(params, n_bands, pixscale=0.03, n_pix=2.0, flux_frac=0.25,
                   q_range=(0.3, 1.0), pa_range=(-0.6 * np.pi, 0.6 * np.pi),
                   sersic_range=(0.8, 6.0), rh_range=(0.02, 0.4)):
    """Lower and upper bounds around ``params`` (n_sources, n_bands + 6), in the
    manner of forcepho's make_bounds (forcepho/superscene.py:805-881): fluxes
    +-5 sigma with a 5% floor on sigma, ra/dec +-n_pix pixels, fixed ranges for
    q, pa, sersic and rh, each widened where needed to contain ``params``."""
    p = np.asarray(params, dtype=np.float64).reshape(-1, n_bands + 6)
    lo, hi = np.empty_like(p), np.empty_like(p)
    f = p[:, :n_bands]
    df = np.maximum(flux_frac * np.abs(f), 1e-3)
    lo[:, :n_bands], hi[:, :n_bands] = f - df, f + df
    dpos = n_pix * pixscale / 3600.0
    dra = dpos / np.cos(np.deg2rad(-27.78))
    lo[:, n_bands], hi[:, n_bands] = p[:, n_bands] - dra, p[:, n_bands] + dra
    lo[:, n_bands + 1], hi[:, n_bands + 1] = p[:, n_bands + 1] - dpos, p[:, n_bands + 1] + dpos
    for j, (a, b) in zip(range(n_bands + 2, n_bands + 6),
                         (q_range, pa_range, sersic_range, rh_range)):
        span = b - a
        lo[:, j] = np.minimum(a, p[:, j] - 0.05 * span)
        hi[:, j] = np.maximum(b, p[:, j] + 0.05 * span)
    return lo.reshape(-1), hi.reshape(-1)


def _param_maps(n_params, dst, src):
    """CSR form (offsets int32 [n_params + 1], indices int64) of the dchi2
    entries of each parameter, from pairs (dst[k], src[k]) grouped by
    parameter in their given order."""
    dst = np.asarray(dst, dtype=np.int64)
    src = np.asarray(src, dtype=np.int64)
    order = np.argsort(dst, kind="stable")
    counts = np.bincount(dst, minlength=n_params)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return off, src[order]


def _device_z(z, n):
    """z as the contiguous float64 CUDA vector of n entries that the fused
    launches read; anything else is refused before a kernel sees it."""
    if not isinstance(z, torch.Tensor) or z.dtype != torch.float64 or not z.is_cuda:
        raise TypeError("z must be a float64 CUDA tensor")
    if z.numel() != n:
        raise ValueError(f"z has {z.numel()} entries, the posterior has {n} parameters")
    return z.contiguous().view(-1)


class _LnpGrad:
    """lnp(z) and d lnp / dz in one launch (fpho_bounded_lnp_grad) from an
    evaluation's chi2 and dchi2, for a bounded transform `tr` and the
    parameters' dchi2 maps."""

    def __init__(self, tr, n_params, dst, src):
        off, idx = _param_maps(n_params, dst, src)
        self.tr, self.n = tr, int(n_params)
        self.off = torch.as_tensor(off, device="cuda")
        self.idx = torch.as_tensor(idx, device="cuda")
        self.work = torch.zeros((self.n + 255) // 256, dtype=torch.float64, device="cuda")
        self.counter = torch.zeros(1, dtype=torch.int32, device="cuda")

    def __call__(self, z, dchi2, chi2, out=None):
        if z.dtype != torch.float64 or not z.is_cuda or not z.is_contiguous():
            raise TypeError("z must be a contiguous float64 CUDA tensor")
        if out is None:
            lnp = torch.empty((), dtype=torch.float64, device="cuda")
            g = torch.empty(self.n, dtype=torch.float64, device="cuda")
        else:
            lnp, g = out
            if (lnp.dtype != torch.float64 or g.dtype != torch.float64 or lnp.numel() != 1
                    or g.numel() != self.n or not g.is_contiguous()):
                raise ValueError("out must be a float64 scalar and a contiguous float64 "
                                 f"vector of {self.n}")
        _lib.call("fpho_bounded_lnp_grad", self.n, z.data_ptr(), self.tr.lower.data_ptr(),
                  self.tr.range.data_ptr(), dchi2.data_ptr(), self.off.data_ptr(),
                  self.idx.data_ptr(), chi2.data_ptr(), chi2.numel(), g.data_ptr(),
                  lnp.data_ptr(), self.work.data_ptr(), self.work.numel(),
                  self.counter.data_ptr(), _stream())
        return lnp, g


class _Bounded:
    """BoundedTransform on the device: q = lower + range * sigmoid(z)."""

    def __init__(self, lower, upper):
        self.lower = torch.as_tensor(np.asarray(lower, dtype=np.float64), device="cuda")
        self.upper = torch.as_tensor(np.asarray(upper, dtype=np.float64), device="cuda")
        self.range = self.upper - self.lower

    def transform(self, z):
        return self.lower + self.range * torch.sigmoid(z)

    def inverse_transform(self, q):
        q = torch.as_tensor(q, dtype=torch.float64, device="cuda")
        return torch.logit((q - self.lower) / self.range)


class DevicePosterior:
    """lnp(z) = lnlike(q(z)) + sum log|dq/dz| for one patch, on the device.

    ``lnprob(z)`` is differentiable through torch autograd (the likelihood
    through :class:`LnLike`); ``lnprob_and_grad(z)`` gives the same value and
    gradient without autograd.  Both enqueue work on the current stream only
    and never synchronize, so a sampler step can be captured in a CUDA graph.
    """

    def __init__(self, patch, lower, upper, table=None, mode="fused"):
        self.ev = PatchEvaluator(patch, table=table, mode=mode)
        self.tr = _Bounded(lower, upper)
        if self.tr.lower.numel() != self.ev.n_params:
            raise ValueError(f"bounds have {self.tr.lower.numel()} entries, the patch has "
                             f"{self.ev.n_params} parameters")
        self.ndim = self.ev.n_params
        # parameter (s, j) of Scene order <- dchi2 entries (band b, source s, k)
        nb, ns = self.ev.n_bands, self.ev.n_sources
        dst, src = [], []
        for s in range(ns):
            for j in range(nb + 6):
                i = s * (nb + 6) + j
                if j < nb:
                    dst.append(i)
                    src.append((j * ns + s) * NPARAMS)
                else:
                    for b in range(nb):
                        dst.append(i)
                        src.append((b * ns + s) * NPARAMS + j - nb + 1)
        self._lnpg = _LnpGrad(self.tr, self.ndim, dst, src)

    def transform(self, z):
        return self.tr.transform(z)

    def inverse_transform(self, q):
        return self.tr.inverse_transform(q)

    def lnprob(self, z):
        s = torch.sigmoid(z)
        q = self.tr.lower + self.tr.range * s
        return LnLike.apply(q, self.ev) + torch.log(self.tr.range * s * (1.0 - s)).sum()

    def lnprob_and_grad(self, z, out=None):
        """(lnp, d lnp / dz) at z: the transform and the proposal build in one
        launch, the evaluation, and lnp with its gradient in one launch
        (written into ``out`` = (lnp, grad) tensors when given)."""
        z = _device_z(z, self.ndim)
        ev = self.ev
        _lib.call("fpho_build_proposal_bounded", ev.table.handle, z.data_ptr(),
                  self.tr.lower.data_ptr(), self.tr.range.data_ptr(), ev.n_sources, ev.n_bands,
                  None, None, None, ev.prop.data_ptr(), _stream())
        ev.evaluate(grad=True)
        return self._lnpg(z, ev.dchi2, ev.chi2, out)

    def _lnprob_and_grad_torch(self, z):
        """The same from torch elementwise operations (the unfused form)."""
        s = torch.sigmoid(z)
        q = self.tr.lower + self.tr.range * s
        jac = self.tr.range * s * (1.0 - s)
        self.ev.run(q, grad=True)
        lnp = self.ev.chi2.sum() * -0.5 + torch.log(jac).sum()
        grad = self.ev.stacked().reshape(-1) * (-0.5 * jac) + (1.0 - 2.0 * s)
        return lnp, grad


class BatchPosterior:
    """lnp(z) summed over the patches of a :class:`forcepho_b200.batch.PatchBatch`
    (independent patches: the gradient of patch k's block depends only on
    patch k), built and evaluated on the device in one batched launch
    sequence."""

    def __init__(self, batch, lowers, uppers, table=None):
        self.batch = batch
        self.table = table if isinstance(table, DeviceSersicTable) else \
            DeviceSersicTable(table or getattr(batch.patches[0], "table", None))
        nb = np.array(batch.n_bands, dtype=np.int64)
        ns = np.array(batch.n_sources, dtype=np.int64)
        npar = ns * (nb + 6)
        self.ndim = int(npar.sum())
        self.tr = _Bounded(np.concatenate(lowers), np.concatenate(uppers))
        if self.tr.lower.numel() != self.ndim:
            raise ValueError("bounds do not match the batch's parameters")
        src_bands = np.repeat(nb, ns).astype(np.int32)
        par_off = np.concatenate([[0], np.cumsum(npar)[:-1]])
        src_off = np.concatenate([po + np.arange(n) * (b + 6)
                                  for po, n, b in zip(par_off, ns, nb)]).astype(np.int64)
        self.src_bands = torch.as_tensor(src_bands, device="cuda")
        self.src_off = torch.as_tensor(src_off, device="cuda")
        n_src = int(ns.sum())
        self.prop = torch.zeros(n_src * SOURCE_BYTES, dtype=torch.uint8, device="cuda")
        self.chi2 = torch.zeros(batch.n_bands_total, dtype=torch.float64, device="cuda")
        self.dchi2 = torch.zeros(batch.n_dchi2, dtype=torch.float32, device="cuda")
        # index maps from the batch's dchi2 layout (per patch: band, source, 7)
        # to the Scene-ordered parameter vector (per patch: source, band | shape)
        flux_dst, flux_src, shape_dst, shape_src = [], [], [], []
        g0 = 0
        for k in range(len(nb)):
            b_, s_ = int(nb[k]), int(ns[k])
            base = int(par_off[k])
            for b in range(b_):
                for s in range(s_):
                    src = g0 + (b * s_ + s) * NPARAMS
                    flux_dst.append(base + s * (b_ + 6) + b)
                    flux_src.append(src)
                    for j in range(1, NPARAMS):
                        shape_dst.append(base + s * (b_ + 6) + b_ + j - 1)
                        shape_src.append(src + j)
            g0 += b_ * s_ * NPARAMS
        cuda = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int64), device="cuda")
        self._lnpg = _LnpGrad(self.tr, self.ndim, flux_dst + shape_dst, flux_src + shape_src)
        self.flux_dst, self.flux_src = cuda(flux_dst), cuda(flux_src)
        # shape gradients: each parameter sums its patch's bands; a padded
        # gather (index n_dchi2 points at an appended zero) keeps the sum
        # deterministic, in band order
        dst = np.asarray(shape_dst, dtype=np.int64)
        srcs = np.asarray(shape_src, dtype=np.int64)
        order = np.argsort(dst, kind="stable")
        dst, srcs = dst[order], srcs[order]
        uniq, first, counts = np.unique(dst, return_index=True, return_counts=True)
        pad = np.full((len(uniq), max(1, int(counts.max()) if len(counts) else 1)),
                      batch.n_dchi2, dtype=np.int64)
        for r, (f, c) in enumerate(zip(first, counts)):
            pad[r, :c] = srcs[f:f + c]
        self.shape_dst, self.shape_src = cuda(uniq), cuda(pad)
        # per-patch sums (one patch per chain in multi-chain sampling): the
        # bands and the parameters of each patch, padded
        self.n_patches = len(nb)
        band_off = np.concatenate([[0], np.cumsum(nb)])
        bpad = np.full((len(nb), int(nb.max())), batch.n_bands_total, dtype=np.int64)
        ppad = np.full((len(nb), int(npar.max())), self.ndim, dtype=np.int64)
        for k in range(len(nb)):
            bpad[k, :nb[k]] = np.arange(band_off[k], band_off[k + 1])
            ppad[k, :npar[k]] = np.arange(par_off[k], par_off[k] + npar[k])
        self.band_pad, self.par_pad = cuda(bpad), cuda(ppad)
        self.par_patch = cuda(np.repeat(np.arange(len(nb)), npar))

    def transform(self, z):
        return self.tr.transform(z)

    def inverse_transform(self, q):
        return self.tr.inverse_transform(q)

    def lnprob_and_grad(self, z, out=None):
        """(lnp, d lnp / dz) at z in five launches: transform and proposals,
        image Gaussians + tiles + reductions of the batch, lnp and gradient
        (written into ``out`` = (lnp, grad) tensors when given)."""
        z = _device_z(z, self.ndim)
        _lib.call("fpho_build_proposal_bounded", self.table.handle, z.data_ptr(),
                  self.tr.lower.data_ptr(), self.tr.range.data_ptr(), self.src_bands.numel(), 0,
                  self.src_bands.data_ptr(), self.src_off.data_ptr(), None, self.prop.data_ptr(),
                  _stream())
        self.batch.evaluate_device(self.prop, self.chi2, self.dchi2, _stream())
        return self._lnpg(z, self.dchi2, self.chi2, out)

    def _lnprob_and_grad_torch(self, z):
        """The same from torch elementwise operations (the unfused form)."""
        s = torch.sigmoid(z)
        q = self.tr.lower + self.tr.range * s
        jac = self.tr.range * s * (1.0 - s)
        self.table.build_proposal_batch(q, self.src_bands, self.src_off, self.prop)
        self.batch.evaluate_device(self.prop, self.chi2, self.dchi2, _stream())
        d = torch.cat([self.dchi2.to(torch.float64), self.chi2.new_zeros(1)])
        gq = torch.empty(self.ndim, dtype=torch.float64, device="cuda")
        gq[self.flux_dst] = d[self.flux_src]
        gq[self.shape_dst] = d[self.shape_src].sum(dim=1)
        lnp = self.chi2.sum() * -0.5 + torch.log(jac).sum()
        return lnp, gq * (-0.5 * jac) + (1.0 - 2.0 * s)

    def lnp_per_patch(self, z):
        """lnp of each patch at z, from the chi2 of the last evaluation (which
        must have been at z)."""
        s = torch.sigmoid(z)
        lj = torch.log(self.tr.range * s * (1.0 - s))
        c = torch.cat([self.chi2, self.chi2.new_zeros(1)])
        lj = torch.cat([lj, lj.new_zeros(1)])
        return c[self.band_pad].sum(dim=1) * -0.5 + lj[self.par_pad].sum(dim=1)


class Leapfrog:
    """Leapfrog integration (unit mass) of Hamiltonian dynamics on a posterior
    with ``lnprob_and_grad(z)`` (or ``lnprob(z)`` through autograd), with
    ``steps_per_graph`` steps captured in one CUDA graph and replayed.

    One step: p += eps/2 g; z += eps p; (lnp, g) = grad(z); p += eps/2 g.
    """

    def __init__(self, posterior, eps=1e-3, steps_per_graph=10, use_autograd=False,
                 use_graph=True):
        self.post = posterior
        self.eps = float(eps)
        self.k = int(steps_per_graph)
        self.use_autograd = use_autograd
        self.use_graph = use_graph
        n = posterior.ndim
        self.z = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.p = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.g = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.lnp = torch.zeros((), dtype=torch.float64, device="cuda")
        self.graph = None

    def _grad(self, z):
        if self.use_autograd:
            zz = z.detach().requires_grad_(True)
            with torch.enable_grad():
                lnp = self.post.lnprob(zz)
                (g,) = torch.autograd.grad(lnp, zz)
            return lnp.detach(), g
        return self.post.lnprob_and_grad(z)

    def _refresh(self):
        if not self.use_autograd and isinstance(self.post, (DevicePosterior, BatchPosterior)):
            self.post.lnprob_and_grad(self.z, out=(self.lnp, self.g))
            return
        lnp, g = self._grad(self.z)
        self.lnp.copy_(lnp)
        self.g.copy_(g)

    def _step(self):
        h = 0.5 * self.eps
        self.p.add_(self.g, alpha=h)
        self.z.add_(self.p, alpha=self.eps)
        self._refresh()
        self.p.add_(self.g, alpha=h)

    def _capture(self):
        saved = [t.clone() for t in (self.z, self.p, self.g, self.lnp)]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(3):  # warm-up outside capture (allocator, kernel attributes)
                self._step()
        torch.cuda.current_stream().wait_stream(side)
        for t, v in zip((self.z, self.p, self.g, self.lnp), saved):
            t.copy_(v)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            for _ in range(self.k):
                self._step()

    def set_state(self, z0, p0):
        self.z.copy_(torch.as_tensor(z0, dtype=torch.float64))
        self.p.copy_(torch.as_tensor(p0, dtype=torch.float64))
        self._refresh()

    def hamiltonian(self):
        return -self.lnp + 0.5 * (self.p * self.p).sum()

    def run(self, n_steps):
        """Advance ``n_steps`` (a multiple of ``steps_per_graph`` when the
        graph is used); enqueued on the current stream, not synchronized."""
        if self.use_graph:
            if n_steps % self.k:
                raise ValueError("n_steps must be a multiple of steps_per_graph")
            if self.graph is None:
                self._capture()
            for _ in range(n_steps // self.k):
                self.graph.replay()
        else:
            for _ in range(n_steps):
                self._step()
