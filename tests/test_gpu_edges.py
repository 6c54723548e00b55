"""GPU: edge cases of the evaluation, each against the oracle (the reference
CPU kernel restated, bit-identical to it) with the bars of the parity tests
(chi2 1e-6 relative; gradient by test_gpu_parity.check_grad):

  * an exposure whose pixels are all masked (ierr = 0), so that some tiles
    have no weight at all;
  * a source far outside the patch, culled from every tile (its gradient is
    exactly zero, as in the reference, where every term is cut at 36);
  * proposals in the reference's clamp branches: sersic below the table
    (one-hot amplitude at the radius nearest rh) and rh < 0 (radius 0);
  * ragged exposures (sides that are not multiples of the 8x8 superpixel,
    with padding) and a single-pixel-wide strip;
  * 64 sources, beyond the reference's 30-source Response limit (against the
    reference's MAXSOURCES=64 build).
"""
import numpy as np
import pytest

from oracle import oracle as O
from test_gpu_parity import CHI2_RTOL, check_grad, gpu_eval

pytestmark = pytest.mark.gpu


def _spec(ns, epb, shapes, npsf=3):
    from forcepho_b200 import synth
    return synth.PatchSpec(n_sources=ns, exposures_per_band=epb, shapes=shapes, n_psf=npsf,
                           psf_sigma=(0.5, 3.0), rot_deg=1.0, scale_frac=0.02,
                           g_range=(0.8, 1.2), mask_frac=0.02, flux_sigma=1.0)


def _check(P, prop, ref=True):
    chi2, dchi2 = gpu_eval(P, prop)
    c32, g32 = O.oracle_evaluate(P, prop, precision="f32")
    np.testing.assert_allclose(chi2, c32, rtol=CHI2_RTOL)
    check_grad(dchi2, g32, P, prop)
    if ref and O.ref_available(P.n_sources):
        cr, gr = O.ref_evaluate(P, prop)
        np.testing.assert_array_equal(cr, c32)
    return chi2, dchi2


def test_fully_masked_exposure():
    from forcepho_b200 import synth
    P = synth.make_patch(_spec(3, [2, 1], [(40, 40)] * 3), seed=21)
    e0, n0 = int(P.exposure_start[1]), int(P.exposure_N[1])
    P.ierr[e0:e0 + n0] = 0.0
    _check(P, P.proposal())


def test_source_off_the_patch():
    from forcepho_b200 import synth
    P = synth.make_patch(_spec(2, [1], [(48, 48)]), seed=22)
    params = P.params.copy()
    params[1, P.n_bands] += 60.0 / 3600.0      # 60 arcsec (2000 px) away in ra
    prop = P.proposal(params)
    chi2, dchi2 = _check(P, prop)
    assert np.all(dchi2[:, 1, :] == 0.0)


def test_clamp_branches():
    from forcepho_b200 import synth
    P = synth.make_patch(_spec(3, [1, 1], [(40, 40)] * 2), seed=23)
    params = P.params.copy()
    nb = P.n_bands
    params[0, nb + 4] = 0.5     # sersic below the table
    params[1, nb + 5] = -0.02   # rh < 0
    prop = P.proposal(params)
    assert np.count_nonzero(prop["mixture_amplitudes"][0]) == 1
    assert prop["mixture_amplitudes"][1][0] == 1.0
    _check(P, prop)


def test_ragged_exposures():
    from forcepho_b200 import synth
    P = synth.make_patch(_spec(2, [2, 1], [(37, 29), (9, 61), (1, 50)]), seed=24)
    assert np.any(P.xpix < 0)   # padding pixels present
    _check(P, P.proposal())


def test_sixty_four_sources():
    from forcepho_b200 import synth
    if not O.ref_available(64):
        pytest.skip("reference CPU kernel (64-source build) not built")
    P = synth.make_patch(_spec(64, [1, 1], [(64, 64)] * 2, npsf=2), seed=25)
    prop = P.proposal()
    chi2, dchi2 = gpu_eval(P, prop)
    cr, gr = O.ref_evaluate(P, prop)
    np.testing.assert_allclose(chi2, cr, rtol=CHI2_RTOL)
    check_grad(dchi2, gr, P, prop)
