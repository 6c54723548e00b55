"""CPU: the host posterior (forcepho_b200.model) on an analytic chi2.

A stand-in proposer returns, per band b, chi2_b = sum_s (flux_sb - a_sb)^2 +
sum_s sum_k w_bk (shape_sk - c_sk)^2 and its exact derivatives in the
(n_bands, n_sources, 7) layout of the evaluation; the posterior must stack
them in Scene order (fluxes per band, then shapes summed over bands), apply
the bounded transform's chain rule and log-Jacobian, cache by position, and
agree with central finite differences."""
import numpy as np
import pytest

from forcepho_b200.model import (BoundedTransform, FastPosterior, Transform, logit, sigmoid,
                                 sigmoid_grad, stack_band_gradients)

NB, NS = 3, 2


class _Scene:
    def set_all_source_params(self, q):
        self.q = np.asarray(q, dtype=np.float64).reshape(NS, NB + 6)

    def get_proposal(self):
        return self.q.copy()


class _Patch:
    n_bands, n_sources = NB, NS
    return_residual = False


class _Proposer:
    def __init__(self, rng):
        self.a = rng.uniform(1, 2, size=(NS, NB))
        self.c = rng.uniform(0.2, 0.8, size=(NS, 6))
        self.w = rng.uniform(0.5, 2.0, size=(NB, 6))
        self.calls = 0

    def evaluate_proposal(self, prop, patch=None, unpack=True):
        self.calls += 1
        f, sh = prop[:, :NB], prop[:, NB:]
        chi2 = np.zeros(NB)
        d = np.zeros((NB, NS, 7))
        for b in range(NB):
            chi2[b] = np.sum((f[:, b] - self.a[:, b]) ** 2) + \
                np.sum(self.w[b] * (sh - self.c) ** 2)
            d[b, :, 0] = 2 * (f[:, b] - self.a[:, b])
            d[b, :, 1:] = 2 * self.w[b] * (sh - self.c)
        out = (chi2, d.astype(np.float32))
        if patch is not None and patch.return_residual:
            out = out + ([np.zeros(4)],)
        return out


def _posterior(sampling=True):
    rng = np.random.default_rng(3)
    lo = np.tile(np.r_[np.zeros(NB), -1, -1, 0.1, -2, 0.5, 0.01], NS)
    hi = np.tile(np.r_[np.full(NB, 4.0), 1, 1, 1.0, 2, 6.0, 1.5], NS)
    prop = _Proposer(rng)
    fp = FastPosterior(prop, _Patch(), scene=_Scene(), lower=lo, upper=hi, sampling=sampling)
    z = rng.normal(scale=0.5, size=lo.size)
    return fp, prop, z


def test_stack_band_gradients_layout():
    d = np.arange(NB * NS * 7, dtype=np.float32).reshape(NB, NS, 7)
    g = stack_band_gradients(d, NB).reshape(NS, NB + 6)
    for s in range(NS):
        assert np.array_equal(g[s, :NB], d[:, s, 0])
        assert np.array_equal(g[s, NB:], d[:, s, 1:].astype(np.float64).sum(axis=0))
    with pytest.raises(ValueError):
        stack_band_gradients(d[:, :, :6], NB)


@pytest.mark.parametrize("sampling", [True, False])
def test_fastposterior_gradient_and_cache(sampling):
    fp, prop, z = _posterior(sampling)
    lnp, g = fp.lnprob_and_grad(z)
    assert prop.calls == 1
    assert fp.lnprob(z.copy()) == lnp and prop.calls == 1        # same position: cached
    q = fp.transform.transform(z)
    chi2, _ = prop.evaluate_proposal(q.reshape(NS, NB + 6))
    want = -0.5 * chi2.sum() + (fp.transform.lndetjac(z) if sampling else 0.0)
    assert lnp == pytest.approx(want, rel=1e-12)
    analytic, numeric = fp.check_grad(z, delta=1e-6)
    np.testing.assert_allclose(analytic, numeric, rtol=2e-5, atol=1e-6)
    nll, ngrad = fp.nll(z)
    assert nll == -lnp and np.array_equal(ngrad, -g)
    assert fp.nll_nograd(z) == -lnp
    assert fp._lnp == lnp and np.array_equal(fp._z, z)


def test_posterior_argument_checks_and_residuals():
    fp, prop, z = _posterior()
    with pytest.raises(ValueError):
        FastPosterior(prop, _Patch(), scene=_Scene())                       # neither
    with pytest.raises(ValueError):
        FastPosterior(prop, _Patch(), scene=_Scene(), transform=Transform(3),
                      lower=[0], upper=[1])                                 # both
    with pytest.raises(ValueError):
        FastPosterior(prop, _Patch(), scene=_Scene(), lower=[0])            # one bound
    with pytest.raises(ValueError):
        FastPosterior(prop, _Patch(), scene=_Scene(), lower=[0], upper=[1], bogus=1)
    res = fp.residuals(fp.transform.transform(z))
    assert len(res) == 1 and fp.patch.return_residual is False


def test_bounded_transform_extremes():
    T = BoundedTransform([0.0, -1.0], [1.0, 3.0])
    z = np.array([-800.0, 800.0])
    q = T.transform(z)
    assert np.all(q >= T.lower) and np.all(q <= T.upper)
    assert np.isfinite(T.lndetjac(z)) and np.all(np.isfinite(T.lndetjac_grad(z)))
    x = np.linspace(-12, 12, 49)   # 1 - s loses digits as s -> 1: keep e^-x above 1e-6
    np.testing.assert_allclose(logit(sigmoid(x)), x, rtol=1e-8, atol=1e-8)
    np.testing.assert_allclose(sigmoid_grad(x), 0.25 / np.cosh(0.5 * x) ** 2, rtol=1e-12)
