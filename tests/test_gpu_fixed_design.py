"""GPU: fixed-source subtraction, the design matrix and the linear flux solve
(forcepho/patches/device_patch.py:113-238, forcepho/fitting.py:573-627).

Bars:
  * design matrix row of each source vs the unit-flux model from the oracle
    (the reference CPU kernel restated, float, on the same patch with zero
    data): |diff| <= 2e-6 |model| + 1e-7 max|model| per pixel;
  * subtract_fixed in blocks, then the active scene evaluated on the
    residual, gives the residual of evaluating every source at once:
    |diff| <= 1e-5 max|data|;
  * the fused device solve (fpho_patch_optimize_fluxes: normal equations
    formed per tile in FP64 without storing the design matrix, Cholesky per
    band) against numpy's optimize_one_band on the device design matrix
    (fpho_patch_design_matrix, the same float rows): precisions 1e-9
    relative, fluxes 1e-9 relative; against numpy on the oracle's design
    matrix: fluxes 1e-6 relative (the float rows differ by rounding);
    at the true shapes the solved fluxes lie within 5 sigma of the true ones
    (sigma from the precision matrix);
  * a source with no pixel in the patch makes its bands' precision matrices
    singular: status 1 and NaN fluxes there, as numpy raises LinAlgError.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _patch(seed=0):
    from forcepho_b200 import synth
    spec = synth.workload_spec("field20")
    spec.shapes = [(48, 48)] * 32
    P = synth.make_patch(spec, seed=seed, render=synth.render_model_gpu)
    return P


def _oracle_design(P, scene):
    """Unit-flux model rows from the f32 oracle on a zero-data copy."""
    prop = scene.get_proposal()
    data = P.data
    P.data = np.zeros_like(data)
    rows = []
    try:
        for i in range(len(prop)):
            q = prop.copy()
            q["fluxes"][:] = 0.0
            q["fluxes"][i, :P.n_bands] = 1.0
            _, _, r = O.oracle_evaluate(P, q, precision="f32", residual=True)
            rows.append(-r.astype(np.float64))
    finally:
        P.data = data
    return np.array(rows)


def test_design_matrix_vs_oracle():
    P = _patch(1)
    P.send_to_device()
    scene = P.set_scene(np.arange(P.n_sources))
    Xes, ys = P.design_matrix(scene)
    X = np.concatenate(Xes, axis=1).astype(np.float64)
    Xo = _oracle_design(P, scene)
    assert X.shape == Xo.shape
    tol = 2e-6 * np.abs(Xo) + 1e-7 * np.abs(Xo).max()
    assert np.all(np.abs(X - Xo) <= tol), float(np.max(np.abs(X - Xo) / (np.abs(Xo).max())))
    np.testing.assert_array_equal(np.concatenate(ys), P.data)
    P.free()


@pytest.mark.parametrize("maxactive", [15, 4])
def test_subtract_fixed_matches_joint_residual(maxactive):
    from forcepho_b200.proposal import GPUProposer
    P = _patch(2)
    ns = P.n_sources
    full = P.set_scene(np.arange(ns))
    P.pack_meta(full)
    P.return_residual = True
    P.free()
    P.send_to_device()
    _, _, r_all = GPUProposer().evaluate_proposal(full.get_proposal(), patch=P, unpack=False)
    fixed, active = np.arange(0, 12), np.arange(12, ns)
    proposer, scene = P.subtract_fixed(fixed, active=active, maxactive=maxactive)
    assert list(scene.source_indices) == list(active)
    np.testing.assert_allclose(P.retrieve_array("data"), _fixed_residual(P, fixed, maxactive),
                               atol=1e-5 * np.abs(P.data).max())
    _, _, r_act = proposer.evaluate_proposal(scene.get_proposal(), patch=P, unpack=False)
    assert np.max(np.abs(r_act - r_all)) <= 1e-5 * np.abs(P.data).max()
    P.free()


def _fixed_residual(P, fixed, maxactive):
    """data minus the model of the fixed sources (oracle, f32, block by block)."""
    res = P.data.astype(np.float64).copy()
    for block in np.array_split(fixed, np.arange(maxactive, len(fixed), maxactive)):
        sc = P.set_scene(block)
        meta = _swap_meta(P, sc)
        data = P.data
        P.data = np.zeros_like(data)
        _, _, r = O.oracle_evaluate(P, sc.get_proposal(), precision="f32", residual=True)
        P.data = data
        _restore_meta(P, meta)
        res += r  # r = -model
    return res


def _swap_meta(P, scene):
    keep = {k: getattr(P, k) for k in ("n_sources", "D", "CW", "crpix", "crval", "psfgauss",
                                       "psfgauss_start")}
    P.pack_meta(scene)
    return keep


def _restore_meta(P, keep):
    for k, v in keep.items():
        setattr(P, k, v)


def test_flux_solve():
    import torch
    from forcepho_b200.fitting import optimize_fluxes, optimize_fluxes_device, optimize_one_band
    P = _patch(3)
    P.send_to_device()
    scene = P.set_scene(np.arange(P.n_sources), params=P.truth)
    fl_h, pr_h = optimize_fluxes(P, scene)     # numpy on the device design matrix
    fl_d, pr_d, st = optimize_fluxes_device(P, scene, return_status=True)
    torch.cuda.synchronize()
    fl_d, pr_d = fl_d.cpu().numpy(), pr_d.cpu().numpy()
    assert np.all(st.cpu().numpy() == 0)
    np.testing.assert_allclose(pr_d, np.array(pr_h), rtol=1e-9)
    np.testing.assert_allclose(fl_d, np.array(fl_h), rtol=1e-9, atol=1e-12)
    # against numpy on the oracle's design matrix
    Xo = _oracle_design(P, scene)
    cuts = np.cumsum(P.band_N_pix[:-1])
    for b, (X, w, y) in enumerate(zip(np.split(Xo, cuts, axis=1), P.split_band("ierr"),
                                      P.split_band("data"))):
        f, _ = optimize_one_band(X, w.astype(np.float64), y.astype(np.float64))
        np.testing.assert_allclose(fl_d[b], np.squeeze(f), rtol=1e-6,
                                   atol=1e-6 * np.abs(f).max())
    # at the true shapes the fluxes are the truth within the noise
    nb = P.n_bands
    for b in range(nb):
        sig = np.sqrt(np.diag(np.linalg.inv(pr_h[b])))
        assert np.all(np.abs(fl_h[b] - P.truth[:, b]) <= 5 * sig + 1e-6 * np.abs(P.truth[:, b]))
    P.free()


def test_flux_solve_singular_band():
    """A source moved far off the patch has a zero design row: every band's
    precision matrix is singular, its fluxes NaN and its status 1."""
    import torch
    from forcepho_b200.fitting import optimize_fluxes_device
    P = _patch(4)
    P.send_to_device()
    params = P.truth.copy()
    params[2, P.n_bands] += 1.0   # ra of source 2: one degree away
    scene = P.set_scene(np.arange(P.n_sources), params=params)
    fl, pr, st = optimize_fluxes_device(P, scene, return_status=True)
    torch.cuda.synchronize()
    st, fl, pr = st.cpu().numpy(), fl.cpu().numpy(), pr.cpu().numpy()
    assert np.all(st == 1) and np.all(np.isnan(fl))
    assert np.all(pr[:, 2, :] == 0) and np.all(pr[:, :, 2] == 0)
    P.free()
