"""The spline layout read by the device proposal builder, pinned on the CPU:
the numpy restatement of bicubic B-spline evaluation (oracle/bspline.py)
against scipy's RectBivariateSpline, which the reference calls
(forcepho/sources.py:623-694), including arguments outside the knot range."""
import numpy as np

from oracle.bspline import bispline


def test_bspline_matches_scipy():
    from forcepho_b200.sources import default_table
    T = default_table()
    tx, ty, c = T.knots_and_coeffs()
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(0.5, 6.5, 40), [tx[3], tx[-4], 6.5, 0.7]])
    ys = np.concatenate([rng.uniform(-0.1, 1.2, 40), [ty[3], ty[-4], 1.3, -0.05]])
    for k in (0, 4, T.n_radii - 1):
        sp = T.splines[k]
        for x, y in zip(xs, ys):
            v, vx, vy = bispline(tx, ty, c[k], x, y)
            sv = float(sp(x, y)[0, 0])
            sx = float(sp(x, y, dx=1)[0, 0])
            sy = float(sp(x, y, dy=1)[0, 0])
            scale = np.abs(c[k]).max()
            assert abs(v - sv) <= 1e-12 * scale, (k, x, y, v, sv)
            assert abs(vx - sx) <= 1e-10 * scale * 100, (k, x, y, vx, sx)
            assert abs(vy - sy) <= 1e-10 * scale * 100, (k, x, y, vy, sy)


def test_bounded_transform_derivatives():
    from forcepho_b200.model import BoundedTransform
    rng = np.random.default_rng(0)
    lo, hi = rng.uniform(-2, 0, 6), rng.uniform(1, 3, 6)
    T = BoundedTransform(lo, hi)
    z = rng.normal(size=6)
    h = 1e-6
    jac = T.jacobian(z)
    for i in range(6):
        dz = np.zeros(6)
        dz[i] = h
        fd = (T.transform(z + dz)[i] - T.transform(z - dz)[i]) / (2 * h)
        assert abs(fd - jac[i]) <= 1e-7 * abs(jac[i])
        fdl = (T.lndetjac(z + dz) - T.lndetjac(z - dz)) / (2 * h)
        assert abs(fdl - T.lndetjac_grad(z)[i]) <= 1e-6
    np.testing.assert_allclose(T.inverse_transform(T.transform(z)), z, rtol=1e-10, atol=1e-12)
