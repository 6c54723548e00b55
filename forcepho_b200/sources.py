"""Sersic mixture amplitudes and the packing of source parameters into
proposals.

:class:`SersicTable` holds the amplitude table of forcepho's Sersic Gaussian
mixtures and evaluates it exactly like ``Galaxy.amplitudes``,
``Galaxy.damplitude_dsersic`` and ``Galaxy.damplitude_drh``
(forcepho/sources.py:623-694): one scipy ``RectBivariateSpline`` (bicubic,
``s=spline_smoothing``) per mixture radius over the (sersic, rh) grid, with the
reference's branches for ``sersic`` below the grid and ``rh < 0``.  The spline
knots and coefficients are exported for the on-device evaluation
(:mod:`forcepho_b200.device_proposal`).

:func:`proposal_from_params` packs a parameter array in the reference's Scene
order ``[flux_1..flux_B, ra, dec, q, pa, sersic, rhalf]`` per source
(forcepho/sources.py:46-97, 526-621) into ``source_struct_dtype``.
"""

import os

import numpy as np
from scipy.interpolate import RectBivariateSpline

from .kernel_limits import MAXRADII
from .proposal import source_struct_dtype

__all__ = ["SersicTable", "Scene", "default_table", "proposal_from_params", "SHAPE_COLS"]

SHAPE_COLS = ["ra", "dec", "q", "pa", "sersic", "rhalf"]
_DEFAULT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                        "sersic_splinedata_large.npz")


class SersicTable:
    """Sersic amplitude splines over a regular (sersic, rh) grid.

    Parameters
    ----------
    ngrid, rgrid : 1-d arrays, the grid of Sersic index and half-light radius
    amplitudes : array (len(ngrid), len(rgrid), n_radii)
    radii : array (n_radii,), mixture radii in arcsec
    spline_smoothing : passed to RectBivariateSpline as ``s`` (None -> 0)
    """

    def __init__(self, ngrid, rgrid, amplitudes, radii, spline_smoothing=None):
        self.ngrid = np.asarray(ngrid, dtype=np.float64)
        self.rgrid = np.asarray(rgrid, dtype=np.float64)
        self.amps = np.asarray(amplitudes, dtype=np.float64)
        self.radii = np.asarray(radii, dtype=np.float64)
        if self.amps.shape != (len(self.ngrid), len(self.rgrid), len(self.radii)):
            raise ValueError("amplitudes must have shape (n_n, n_r, n_radii)")
        if len(self.radii) > MAXRADII:
            raise ValueError(f"at most {MAXRADII} mixture radii")
        s = 0 if spline_smoothing is None else spline_smoothing
        self.splines = [RectBivariateSpline(self.ngrid, self.rgrid, self.amps[:, :, i], s=s)
                        for i in range(len(self.radii))]
        self.sersic_range = (self.ngrid.min(), self.ngrid.max())
        self.rh_range = (self.rgrid.min(), self.rgrid.max())

    @classmethod
    def from_file(cls, path, spline_smoothing=None):
        """A table from forcepho's spline-data HDF5 file (datasets nsersic,
        rh, amplitudes of shape (n_grid, n_radii), radii; read as
        forcepho/sources.py:623-645 does) or from this package's ``.npz``
        form (ngrid, rgrid, amplitudes (n_n, n_r, n_radii), radii)."""
        if str(path).endswith(".npz"):
            d = np.load(path)
            return cls(d["ngrid"], d["rgrid"], d["amplitudes"], d["radii"], spline_smoothing)
        from . import h5lite
        with h5lite.File(path) as f:
            n = np.asarray(f["nsersic"][:], dtype=np.float64)
            r = np.asarray(f["rh"][:], dtype=np.float64)
            A = np.asarray(f["amplitudes"][:])
            radii = np.asarray(f["radii"][:], dtype=np.float64)
        ngrid, rgrid = np.unique(n), np.unique(r)
        amps = np.stack([A[:, i].reshape(len(ngrid), len(rgrid)) for i in range(A.shape[1])], -1)
        return cls(ngrid, rgrid, amps, radii, spline_smoothing)

    @property
    def n_radii(self):
        return len(self.radii)

    @property
    def rad2(self):
        return (self.radii ** 2).astype(np.float32)

    def amplitudes(self, sersic, rhalf):
        if sersic < self.sersic_range[0]:
            amp = np.zeros(self.n_radii)
            amp[np.argmin(np.abs(rhalf - self.radii))] = 1.0
        elif rhalf < 0:
            amp = np.zeros(self.n_radii)
            amp[0] = 1.0
        else:
            amp = np.array([float(sp(sersic, rhalf)[0, 0]) for sp in self.splines])
        return amp

    def damplitude_dsersic(self, sersic, rhalf):
        if sersic < self.sersic_range[0] or rhalf < 0:
            return np.zeros(self.n_radii)
        return np.array([float(sp(sersic, rhalf, dx=1)[0, 0]) for sp in self.splines])

    def damplitude_drh(self, sersic, rhalf):
        if sersic < self.sersic_range[0] or rhalf < 0:
            return np.zeros(self.n_radii)
        return np.array([float(sp(sersic, rhalf, dy=1)[0, 0]) for sp in self.splines])

    def amplitudes_many(self, sersic, rhalf):
        """(amplitudes, d/dsersic, d/drh), each (n, n_radii), for arrays of
        sources: the values ``amplitudes`` / ``damplitude_dsersic`` /
        ``damplitude_drh`` give one source at a time (the splines are
        evaluated at all points in one call each, with identical results),
        with the same branches for sersic below the grid and rh < 0."""
        n = np.atleast_1d(np.asarray(sersic, dtype=np.float64))
        r = np.atleast_1d(np.asarray(rhalf, dtype=np.float64))
        m = len(n)
        amp = np.zeros((m, self.n_radii))
        dn = np.zeros((m, self.n_radii))
        dr = np.zeros((m, self.n_radii))
        low = n < self.sersic_range[0]
        neg = ~low & (r < 0)
        ok = ~low & ~neg
        if ok.any():
            for i, sp in enumerate(self.splines):
                amp[ok, i] = sp(n[ok], r[ok], grid=False)
                dn[ok, i] = sp(n[ok], r[ok], dx=1, grid=False)
                dr[ok, i] = sp(n[ok], r[ok], dy=1, grid=False)
        for j in np.flatnonzero(low):
            amp[j, np.argmin(np.abs(r[j] - self.radii))] = 1.0
        amp[neg, 0] = 1.0
        return amp, dn, dr

    def knots_and_coeffs(self):
        """(tx, ty, coeffs[n_radii, len(tx)-4, len(ty)-4]) of the bicubic
        splines; all radii share the knot vectors."""
        tx, ty = self.splines[0].get_knots()
        for sp in self.splines[1:]:
            a, b = sp.get_knots()
            if not (np.array_equal(a, tx) and np.array_equal(b, ty)):
                raise ValueError("splines do not share knots")
        nc = (len(tx) - 4, len(ty) - 4)
        c = np.stack([sp.get_coeffs().reshape(nc) for sp in self.splines])
        return tx, ty, c


_default_table = None


def default_table():
    """The table extracted from forcepho's ``sersic_splinedata_large.h5``
    (sersic 0.8..6.2, rh 0..1 arcsec, 9 radii)."""
    global _default_table
    if _default_table is None:
        d = np.load(_DEFAULT)
        _default_table = SersicTable(d["ngrid"], d["rgrid"], d["amplitudes"], d["radii"])
    return _default_table


def proposal_from_params(params, n_bands, table=None, per_source=None):
    """Pack parameters of shape (n_sources, n_bands + 6), in Scene order, into
    a ``source_struct_dtype`` array (as ``Galaxy.proposal``,
    forcepho/sources.py:607-621).  The amplitude splines are evaluated for all
    sources in one call per radius, or, with `per_source` (the default for one
    or two sources, where it is faster), one source at a time as the
    reference does; the bytes are the same either way."""
    table = table or default_table()
    params = np.asarray(params, dtype=np.float64).reshape(-1, n_bands + 6)
    out = np.zeros(len(params), dtype=source_struct_dtype)
    nr = table.n_radii
    out["fluxes"][:, :n_bands] = params[:, :n_bands]
    for k, name in enumerate(["ra", "dec", "q", "pa", "nsersic", "rh"]):
        out[name] = params[:, n_bands + k]
    if per_source is None:
        per_source = len(params) <= 2
    if per_source:
        for i, p in enumerate(params):
            n, rh = p[n_bands + 4], p[n_bands + 5]
            out["mixture_amplitudes"][i, :nr] = table.amplitudes(n, rh)
            out["damplitude_drh"][i, :nr] = table.damplitude_drh(n, rh)
            out["damplitude_dnsersic"][i, :nr] = table.damplitude_dsersic(n, rh)
        return out
    amp, dn, dr = table.amplitudes_many(params[:, n_bands + 4], params[:, n_bands + 5])
    out["mixture_amplitudes"][:, :nr] = amp
    out["damplitude_drh"][:, :nr] = dr
    out["damplitude_dnsersic"][:, :nr] = dn
    return out


class Scene:
    """The map between the flat parameter vector of the active sources and
    their proposal (forcepho/sources.py:28-97: ``set_all_source_params``,
    ``get_all_source_params``, ``get_proposal``), for ``n_sources`` Sersic
    galaxies of ``n_bands`` fluxes each, in Scene order."""

    def __init__(self, n_sources, n_bands, table=None, params=None, per_source=None):
        self.n_sources, self.n_bands = int(n_sources), int(n_bands)
        self.table = table or default_table()
        self.per_source = per_source       # see proposal_from_params
        self.n_params_per_source = self.n_bands + 6
        self.params = np.zeros((self.n_sources, self.n_params_per_source))
        if params is not None:
            self.set_all_source_params(params)

    def __len__(self):
        return self.n_sources

    def set_all_source_params(self, Theta):
        self.params[:] = np.asarray(Theta, dtype=np.float64).reshape(self.params.shape)

    def get_all_source_params(self, active=True):
        return self.params.reshape(-1).copy()

    def get_proposal(self, active=True):
        return proposal_from_params(self.params, self.n_bands, self.table,
                                    per_source=self.per_source)
