"""Posterior objects over the proposal evaluation (host side).

The drop-in surface of forcepho/model.py: :class:`Posterior` with
``lnprob`` / ``lnprob_grad`` / ``lnprob_and_grad`` / ``nll`` /
``nll_nograd`` / ``check_grad`` / ``make_transform`` (model.py:40-257),
:class:`FastPosterior` with ``evaluate``, ``stack_grad`` and ``residuals``
(model.py:260-405), the ``GPUPosterior`` alias, and the parameter transforms
:class:`Transform` / :class:`BoundedTransform` with ``sigmoid``, ``logit``
and ``sigmoid_grad`` (model.py:555-637).  Names, arguments and returned
values are the reference's, so its fitting code runs on these objects.

The implementation is this package's own:

* one evaluation produces an immutable :class:`_Point` (z, q, lnp, its
  gradient); the accessors answer from the last point when called again at
  the same z, which is what samplers and optimisers do (value and gradient at
  one position, then a new position);
* the bounded transform is written around the logistic s = 1/(1+e^-z):
  q = lo + (hi-lo) s, dq/dz = (hi-lo) s (1-s) with 1-s = sigmoid(-z), and
  log|dq/dz| uses log s = -softplus(-z), log(1-s) = -softplus(z), finite for
  any z;
* the per-band gradient of the evaluation, (n_bands, n_sources, 7), becomes
  the Scene-ordered vector by array operations (:func:`stack_band_gradients`).

The proposer is a :class:`forcepho_b200.proposal.GPUProposer`; the scene is any
object with ``set_all_source_params`` and ``get_proposal`` (see
:class:`forcepho_b200.sources.Scene`).  The device-resident posterior of the
differentiable form is :class:`forcepho_b200.autograd.DevicePosterior`.
"""

from dataclasses import dataclass

import numpy as np
from scipy.special import expit

from .kernel_limits import NPARAMS

__all__ = ["Posterior", "FastPosterior", "GPUPosterior", "Transform", "BoundedTransform",
           "sigmoid", "logit", "sigmoid_grad", "stack_band_gradients"]


# ------------------------------------------------------------------ transforms
def sigmoid(x):
    """The logistic function 1 / (1 + exp(-x))."""
    return expit(x)


def logit(y):
    """Inverse of :func:`sigmoid`: log(y / (1 - y))."""
    y = np.asarray(y, dtype=np.float64)
    return np.log(y) - np.log1p(-y)


def sigmoid_grad(z):
    """d sigmoid / dz = s (1 - s), with 1 - s taken as sigmoid(-z) (no
    cancellation when s is near 1)."""
    return expit(z) * expit(-z)


def _softplus(x):
    """log(1 + e^x) without overflow."""
    return np.logaddexp(0.0, x)


class Transform:
    """The identity map between the sampler's coordinates z and the
    parameters q (unit Jacobian)."""

    def __init__(self, ndim):
        self.ndim = ndim

    def transform(self, z):
        return np.array(z, dtype=np.float64)

    def inverse_transform(self, Theta):
        return np.array(Theta, dtype=np.float64)

    def jacobian(self, z):
        return np.ones(np.shape(z)[-1] if np.ndim(z) else 1)

    def lndetjac(self, z):
        return float(np.sum(np.log(np.abs(self.jacobian(z)))))

    def lndetjac_grad(self, z):
        return np.zeros(np.shape(z)[-1] if np.ndim(z) else 1)


class BoundedTransform(Transform):
    """q = lower + (upper - lower) * sigmoid(z), element by element: every z
    maps inside the open box (lower, upper) (forcepho/model.py:596-637)."""

    def __init__(self, lower, upper):
        lo = np.atleast_1d(np.asarray(lower, dtype=np.float64))
        hi = np.atleast_1d(np.asarray(upper, dtype=np.float64))
        if lo.shape != hi.shape:
            raise ValueError(f"lower {lo.shape} and upper {hi.shape} differ in shape")
        self.lower, self.upper = lo, hi
        self.ndim = lo.size

    @property
    def range(self):
        return self.upper - self.lower

    def transform(self, z):
        return self.lower + self.range * expit(z)

    def inverse_transform(self, Theta):
        return logit((np.asarray(Theta, dtype=np.float64) - self.lower) / self.range)

    def jacobian(self, z):
        """dq/dz, the diagonal of the Jacobian."""
        return self.range * sigmoid_grad(z)

    def lndetjac(self, z):
        """log |det dq/dz| = sum(log range + log s + log(1 - s))."""
        z = np.asarray(z, dtype=np.float64)
        return float(np.sum(np.log(np.abs(self.range)) - _softplus(-z) - _softplus(z)))

    def lndetjac_grad(self, z):
        """d log|det dq/dz| / dz = 1 - 2 s."""
        return 1.0 - 2.0 * expit(z)


# ------------------------------------------------------------------ gradients
def stack_band_gradients(dchi2, n_bands):
    """Per-band d chi2 / d(flux, ra, dec, q, pa, sersic, rh), shape
    (n_bands, n_sources, 7), as one Scene-ordered vector: per source the
    flux derivatives band by band, then the six shape derivatives summed over
    bands (each band constrains the same shape).  float64."""
    d = np.asarray(dchi2, dtype=np.float64)
    if d.ndim != 3 or d.shape[0] != n_bands or d.shape[2] != NPARAMS:
        raise ValueError(f"expected (n_bands={n_bands}, n_sources, {NPARAMS}), got {d.shape}")
    fluxes = d[:, :, 0].T                   # (n_sources, n_bands)
    shapes = d[:, :, 1:].sum(axis=0)        # (n_sources, 6)
    return np.concatenate([fluxes, shapes], axis=1).reshape(-1)


# ------------------------------------------------------------------ posteriors
@dataclass(frozen=True)
class _Point:
    """One evaluated position: sampler coordinates z, parameters q, the log
    posterior and its gradient with respect to z."""
    z: np.ndarray
    q: np.ndarray
    lnp: float
    lnp_grad: np.ndarray


class Posterior:
    """Log posterior in the sampler's coordinates z, with the parameters
    q = transform(z).  Subclasses implement :meth:`evaluate`, which computes
    lnp and d lnp / dz at z and records them with :meth:`_remember`.

    Keyword arguments: either ``transform`` (a :class:`Transform`) or
    ``lower`` and ``upper`` (a :class:`BoundedTransform` is made from them);
    nothing else is accepted.
    """

    def __init__(self, **kwargs):
        transform = kwargs.pop("transform", None)
        lower, upper = kwargs.pop("lower", None), kwargs.pop("upper", None)
        if kwargs:
            raise ValueError(f"Posterior got argument(s) it does not understand: "
                             f"{sorted(kwargs)}")
        bounds = lower is not None and upper is not None
        if bool(transform) == bounds or (lower is None) != (upper is None):
            raise ValueError('give either "transform" or both "lower" and "upper"')
        self.transform = transform if transform is not None else BoundedTransform(lower, upper)
        self.ncall = 0
        self.ndof = 1.0
        self._point = None
        self._lnpriorfn = None

    # ---- caching
    def _remember(self, z, q, lnp, grad):
        self._point = _Point(np.array(z, dtype=np.float64, copy=True), np.asarray(q),
                             float(lnp), np.asarray(grad, dtype=np.float64))
        return self._point

    def _at(self, z):
        p = self._point
        if p is None or np.shape(z) != p.z.shape or not np.array_equal(z, p.z):
            self.evaluate(z)
            p = self._point
        return p

    # attributes of the reference's objects, read from the last point
    @property
    def _z(self):
        return None if self._point is None else self._point.z

    @property
    def _q(self):
        return None if self._point is None else self._point.q

    @property
    def _lnp(self):
        return None if self._point is None else self._point.lnp

    @property
    def _lnp_grad(self):
        return None if self._point is None else self._point.lnp_grad

    # ---- the interface samplers and optimisers call
    def evaluate(self, z):
        raise NotImplementedError

    def lnprob(self, z):
        return self._at(z).lnp

    def lnprob_grad(self, z):
        return self._at(z).lnp_grad

    def lnprob_and_grad(self, z):
        p = self._at(z)
        return p.lnp, p.lnp_grad

    def nll(self, z):
        """(-lnp / ndof, -d lnp/dz / ndof): the objective of a minimiser."""
        p = self._at(z)
        return -p.lnp / self.ndof, -p.lnp_grad / self.ndof

    def nll_nograd(self, z):
        return -self._at(z).lnp / self.ndof

    def lnprior(self, q):
        """(ln prior, d ln prior / dq) from the prior function, or (0, 0)."""
        if self._lnpriorfn is None:
            return 0.0, 0.0
        return self._lnpriorfn(q)

    def make_transform(self, z):
        """q = transform(z); keeps dq/dz, log|dq/dz| and its gradient at z
        (``_jacobian``, ``_lndetjac``, ``_lndetjac_grad``) for the chain rule."""
        T = self.transform
        if T is None:
            self._jacobian, self._lndetjac, self._lndetjac_grad = 1.0, 0.0, 0.0
            return np.array(z, dtype=np.float64)
        self._jacobian = T.jacobian(z)
        self._lndetjac = T.lndetjac(z)
        self._lndetjac_grad = T.lndetjac_grad(z)
        return T.transform(z)

    def residuals(self, z):
        raise NotImplementedError

    def check_grad(self, z, delta=1e-5):
        """(analytic d lnp/dz, central finite differences with step `delta`)."""
        z0 = np.array(z, dtype=np.float64)
        analytic = np.array(self.lnprob_grad(z0), copy=True)
        steps = np.broadcast_to(np.asarray(delta, dtype=np.float64), z0.shape)
        numeric = np.empty_like(z0)
        for i in range(z0.size):
            e = np.zeros_like(z0)
            e[i] = steps[i]
            numeric[i] = (self.lnprob(z0 + e) - self.lnprob(z0 - e)) / (2.0 * steps[i])
        return analytic, numeric


class FastPosterior(Posterior):
    """lnp(z) = -chi2(q)/2 + ln prior(q) [+ log|dq/dz| when ``sampling``],
    chi2 and its gradient from the proposer's evaluation of the scene's
    proposal on the patch (forcepho/model.py:260-405)."""

    def __init__(self, proposer, patch, scene=None, lnprior=None, transform=None, name="",
                 print_interval=1000, verbose=False, debug=False, logging=False, sampling=True,
                 **kwargs):
        super().__init__(transform=transform, **kwargs)
        self.proposer = proposer
        self.patch = patch
        self.scene = scene if scene is not None else patch.scene
        self._lnpriorfn = lnprior
        self.sampling = sampling
        self.name = name
        self.print_interval = print_interval
        self.verbose, self.debug, self.logging = verbose, debug, logging
        self._residuals = None
        if logging:
            self.pos_history, self.lnp_history, self.grad_history = [], [], []

    def _chi2(self, q, **kw):
        """Set the scene to q, evaluate its proposal; the proposer's output."""
        self.scene.set_all_source_params(q)
        return self.proposer.evaluate_proposal(self.scene.get_proposal(), patch=self.patch, **kw)

    def evaluate(self, z):
        q = self.make_transform(z)
        out = self._chi2(q)
        chi2, dchi2 = out[0], out[1]
        if len(out) > 2:
            self._residuals = out[2]
        lnlike = -0.5 * float(np.sum(np.asarray(chi2, dtype=np.float64)))
        dlnlike = -0.5 * self.stack_grad(dchi2)
        lnpr, dlnpr = self.lnprior(q)
        lnp = lnlike + lnpr
        grad = (dlnlike + dlnpr) * self._jacobian     # chain rule, dq/dz diagonal
        if self.sampling:
            lnp = lnp + self._lndetjac
            grad = grad + self._lndetjac_grad
        self.ncall += 1
        if self.logging:
            self._lnlike, self._lnlike_grad = lnlike, dlnlike
            self._lnprior, self._lnprior_grad = lnpr, dlnpr
            self.pos_history.append(np.array(z, copy=True))
            self.lnp_history.append(lnlike)
            self.grad_history.append(dlnlike)
        if self.verbose and self.ncall % self.print_interval == 0:
            print(f"{self.name} call {self.ncall}: lnlike {lnlike:.6g}")
        self._remember(z, q, lnp, grad)

    def stack_grad(self, chi2_derivs):
        """(n_bands, n_sources, 7) d chi2 -> the Scene-ordered gradient vector
        (:func:`stack_band_gradients`)."""
        return stack_band_gradients(chi2_derivs, self.patch.n_bands)

    def residuals(self, q, unpack=True):
        """The residual images (data - model) at parameters q."""
        keep = self.patch.return_residual
        self.patch.return_residual = True
        try:
            self._residuals = self._chi2(q, unpack=unpack)[2]
        finally:
            self.patch.return_residual = keep
        return self._residuals


class GPUPosterior(FastPosterior):
    """The reference's name for the same posterior (forcepho/model.py:408)."""
