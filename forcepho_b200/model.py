"""Posterior objects over the proposal evaluation.

Mirrors forcepho/model.py: :class:`Posterior` (caching, ``lnprob``,
``lnprob_grad``, ``lnprob_and_grad``, ``nll``, ``check_grad``,
``make_transform``; model.py:40-257), :class:`FastPosterior` (``evaluate``
and ``stack_grad``; model.py:260-405) and the parameter transforms
:class:`Transform` / :class:`BoundedTransform` (model.py:571-637).  The
proposer is a :class:`forcepho_b200.proposal.GPUProposer`; the scene is any
object with ``set_all_source_params`` and ``get_proposal`` (see
:class:`forcepho_b200.sources.Scene`).
"""

import numpy as np
from scipy.special import expit

from .kernel_limits import NPARAMS

__all__ = ["Posterior", "FastPosterior", "GPUPosterior", "Transform", "BoundedTransform",
           "sigmoid", "logit", "sigmoid_grad"]


class Posterior:
    """Caching base class (forcepho/model.py:40-257)."""

    def __init__(self, **kwargs):
        self.ncall = 0
        self.ndof = 1.0
        if (np.any(kwargs.get('lower')) and np.any(kwargs.get('upper'))) == \
                bool(kwargs.get('transform')):
            raise ValueError('Must specify either "transform" or ("lower","upper")')
        transform = kwargs.pop('transform', None)
        if transform is not None:
            self.transform = transform
        else:
            self.transform = BoundedTransform(kwargs.pop('lower'), kwargs.pop('upper'))
        if kwargs:
            raise ValueError(f'Passed argument(s) {list(kwargs.keys())} to Posterior that '
                             'were not understood')

    def evaluate(self, z):
        raise NotImplementedError

    def lnprob(self, z):
        if np.any(z != self._z):
            self.evaluate(z)
        return self._lnp

    def lnprob_grad(self, z):
        if np.any(z != self._z):
            self.evaluate(z)
        return self._lnp_grad

    def lnprob_and_grad(self, z):
        if np.any(z != self._z):
            self.evaluate(z)
        return self._lnp, self._lnp_grad

    def lnprior(self, q):
        if self._lnpriorfn is None:
            return 0.0, 0.0
        return self._lnpriorfn(q)

    def make_transform(self, z):
        if self.transform is not None:
            self._jacobian = self.transform.jacobian(z)
            self._lndetjac = self.transform.lndetjac(z)
            self._lndetjac_grad = self.transform.lndetjac_grad(z)
            return self.transform.transform(z)
        self._jacobian = 1.
        self._lndetjac = 0
        self._lndetjac_grad = 0
        return np.array(z)

    def nll(self, z):
        if np.any(z != self._z):
            self.evaluate(z)
        return -self._lnp / self.ndof, -self._lnp_grad / self.ndof

    def nll_nograd(self, z):
        if np.any(z != self._z):
            self.evaluate(z)
        return -self._lnp / self.ndof

    def residuals(self, z):
        raise NotImplementedError

    def check_grad(self, z, delta=1e-5):
        """Central finite differences against the analytic gradient."""
        z0 = np.array(z, dtype=np.float64).copy()
        dlnp = self.lnprob_grad(z0)
        delta = np.zeros_like(dlnp) + delta
        dlnp_num = np.zeros(len(z0), dtype=np.float64)
        for i, dp in enumerate(delta):
            theta = z0.copy()
            theta[i] -= dp
            imlo = self.lnprob(theta.copy())
            theta[i] += 2 * dp
            imhi = self.lnprob(theta.copy())
            dlnp_num[i] = (imhi - imlo) / (2 * dp)
        return dlnp, dlnp_num


class FastPosterior(Posterior):
    """lnp = -chi2/2 (+ prior, + log|dq/dz| when sampling) from the GPU proposer
    (forcepho/model.py:260-405)."""

    def __init__(self, proposer, patch, scene=None, lnprior=None, transform=None, name="",
                 print_interval=1000, verbose=False, debug=False, logging=False, sampling=True,
                 **kwargs):
        super().__init__(transform=transform, **kwargs)
        self.proposer = proposer
        self.patch = patch
        self.scene = scene if scene else self.patch.scene
        self._lnpriorfn = lnprior
        self.sampling = sampling
        self.ncall = 0
        self._z = -99
        self._q = -99
        self.mhalf = np.array(-0.5, dtype=np.float64)
        self.debug, self.logging, self.verbose = debug, logging, verbose
        self.print_interval, self.name = print_interval, name
        if self.logging:
            self.pos_history, self.lnp_history, self.grad_history = [], [], []

    def evaluate(self, z):
        q = self.make_transform(z)
        self.scene.set_all_source_params(q)
        proposal = self.scene.get_proposal()
        lpr, lpr_grad = self.lnprior(q)
        ret = self.proposer.evaluate_proposal(proposal, patch=self.patch)
        if len(ret) == 3:
            chi2, chi2_derivs, self._residuals = ret
        else:
            chi2, chi2_derivs = ret
        ll = self.mhalf * np.array(chi2.astype(np.float64).sum(), dtype=np.float64)
        ll_grad = self.mhalf * self.stack_grad(chi2_derivs)
        self.ncall += 1
        if self.logging:
            self._lnlike, self._lnlike_grad = ll, ll_grad
            self._lnprior, self._lnprior_grad = lpr, lpr_grad
            self.pos_history.append(z)
            self.lnp_history.append(ll)
            self.grad_history.append(ll_grad)
        self._lnp = ll + lpr
        self._lnp_grad = (ll_grad + lpr_grad) * self._jacobian
        self._q, self._z = q, z
        if self.sampling:
            self._lnp += self._lndetjac
            self._lnp_grad += self._lndetjac_grad
        if self.verbose and np.mod(self.ncall, self.print_interval) == 0:
            print(f"-------\n {self.name} @ {self.ncall}\nq: {q}\nlnlike: {ll}")

    def stack_grad(self, chi2_derivs):
        """(n_bands, n_sources, 7) -> per source [flux_1..flux_B, ra, dec, q, pa,
        sersic, rh]: fluxes per band, shape gradients summed over bands."""
        nsources, nbands = self.patch.n_sources, self.patch.n_bands
        grads = np.zeros([nsources, nbands + (NPARAMS - 1)], dtype=np.float64)
        for band, derivs in enumerate(chi2_derivs):
            grads[:, nbands:] += derivs[:, 1:]
            grads[:, band] += derivs[:, 0]
        return grads.reshape(-1)

    def residuals(self, q, unpack=True):
        orig = self.patch.return_residual
        self.patch.return_residual = True
        self.scene.set_all_source_params(q)
        proposal = self.scene.get_proposal()
        ret = self.proposer.evaluate_proposal(proposal, patch=self.patch, unpack=unpack)
        self._residuals = ret[2]
        self.patch.return_residual = orig
        return self._residuals


class GPUPosterior(FastPosterior):
    """Alias kept for compatibility with the reference."""
    pass


# ------------------------------------------------------------------ transforms
def sigmoid(x):
    return expit(x)


def logit(y):
    return -np.log(1. / y - 1.)


def sigmoid_grad(z):
    return (0.5 / np.cosh(0.5 * z)) ** 2


class Transform:

    def __init__(self, ndim):
        self.ndim = ndim

    def transform(self, z):
        return np.array(z)

    def jacobian(self, z):
        return np.ones(len(z))

    def lndetjac(self, z):
        return np.log(np.abs(np.prod(self.jacobian(z))))

    def lndetjac_grad(self, z):
        return np.zeros(len(z))

    def inverse_transform(self, Theta):
        return np.array(Theta)


class BoundedTransform(Transform):
    """q = lower + (upper - lower) * sigmoid(z) (forcepho/model.py:596-637)."""

    def __init__(self, lower, upper):
        self.lower = np.atleast_1d(lower)
        self.upper = np.atleast_1d(upper)
        assert len(self.upper) == len(self.lower)
        self.ndim = len(self.upper)

    @property
    def range(self):
        return self.upper - self.lower

    def transform(self, z):
        return self.lower + sigmoid(z) * self.range

    def jacobian(self, z):
        return self.range * sigmoid_grad(z)

    def lndetjac(self, z):
        return np.sum(np.log(np.abs(self.jacobian(z))))

    def lndetjac_grad(self, z):
        return 1 - 2.0 * sigmoid(z)

    def inverse_transform(self, Theta):
        return logit((Theta - self.lower) / self.range)
