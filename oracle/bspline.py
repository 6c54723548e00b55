"""Oracle (test infrastructure only): bicubic B-spline evaluation in numpy.

The reference evaluates the Sersic mixture amplitudes and their derivatives
with scipy's ``RectBivariateSpline`` (forcepho/sources.py:623-694; a
third-party dependency absent from the reference tree, scipy 1.x, whose
``__call__`` is FITPACK's ``bispev`` / ``parder``).  This restates the
published algorithm: de Boor's recursion for the four non-zero cubic
B-splines on the knot interval holding x, the derivative identity
B'_{i,3}(x) = 3 (B_{i,2}(x) / (t_{i+3} - t_i) - B_{i+1,2}(x) / (t_{i+4} - t_{i+1})),
and FITPACK's clamping of arguments to [t[3], t[n-4]].  The coefficient
layout it assumes -- c[(ix) * (len(ty) - 4) + iy], as ``get_coeffs()``
returns it -- is the one the device kernel reads, so agreement with scipy
pins that layout.  Tests call :func:`bispline` and compare with scipy.
"""

import numpy as np

__all__ = ["cubic_basis", "bispline"]


def cubic_basis(t, x):
    """(l, B[4], dB[4]) at scalar x for knot vector t (degree 3)."""
    t = np.asarray(t, dtype=np.float64)
    n = len(t)
    x = min(max(float(x), t[3]), t[n - 4])
    l = int(np.searchsorted(t, x, side="right")) - 1
    l = min(max(l, 3), n - 5)
    # N[r] holds B_{l-j+r, j} for r = 0..j (Cox-de Boor, degree by degree)
    N = np.zeros(4)
    N[0] = 1.0
    N2 = None
    for j in range(1, 4):
        new = np.zeros(4)
        for r in range(j + 1):
            i = l - j + r  # B_{i,j}
            val = 0.0
            if r >= 1:      # B_{i,j-1} = N[r-1]
                d = t[i + j] - t[i]
                if d != 0:
                    val += (x - t[i]) / d * N[r - 1]
            if r <= j - 1:  # B_{i+1,j-1} = N[r]
                d = t[i + j + 1] - t[i + 1]
                if d != 0:
                    val += (t[i + j + 1] - x) / d * N[r]
            new[r] = val
        N = new
        if j == 2:
            N2 = N[:3].copy()
    B = N.copy()
    dB = np.zeros(4)
    for r in range(4):
        i = l - 3 + r
        b0 = N2[r - 1] if r >= 1 else 0.0
        b1 = N2[r] if r <= 2 else 0.0
        d0, d1 = t[i + 3] - t[i], t[i + 4] - t[i + 1]
        dB[r] = 3.0 * ((b0 / d0 if d0 != 0 else 0.0) - (b1 / d1 if d1 != 0 else 0.0))
    return l, B, dB


def bispline(tx, ty, c, x, y):
    """(value, d/dx, d/dy) of the bicubic spline with knots tx, ty and
    coefficients c (flat, or shaped (len(tx)-4, len(ty)-4)) at (x, y)."""
    ncy = len(ty) - 4
    c = np.asarray(c, dtype=np.float64).reshape(len(tx) - 4, ncy)
    lx, Bx, dBx = cubic_basis(tx, x)
    ly, By, dBy = cubic_basis(ty, y)
    blk = c[lx - 3:lx + 1, ly - 3:ly + 1]
    return float(Bx @ blk @ By), float(dBx @ blk @ By), float(Bx @ blk @ dBy)
