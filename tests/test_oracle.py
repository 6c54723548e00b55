"""The oracle is pinned before it is trusted: its float restatement must be
bit-identical to the reference CPU kernel (committed golden vectors, and the
kernel itself when oracle/_ref is built), and its FP64 restatement must agree
with the reference's FP64 slow path."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden
from oracle import oracle as O
from forcepho_b200 import synth


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_f32_oracle_bitexact_vs_golden_reference(name):
    P, prop, d = load_golden(name)
    chi2, dchi2 = O.oracle_evaluate(P, prop)
    assert np.array_equal(chi2, d["ref_chi2"])
    assert np.array_equal(dchi2, d["ref_dchi2"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_f64_oracle_vs_golden_slow_path(name):
    P, prop, d = load_golden(name)
    chi2, dchi2 = O.oracle_evaluate(P, prop, precision="f64", cutoff=False)
    np.testing.assert_allclose(chi2, d["slow_chi2"], rtol=1e-10, atol=1e-8)
    scale = np.abs(d["slow_dchi2"]).max(axis=(0, 1), keepdims=True)
    np.testing.assert_allclose(dchi2, d["slow_dchi2"], rtol=1e-8, atol=1e-10 * scale.max())


def _small_spec(ns, epb, side, npsf=2):
    return synth.PatchSpec(n_sources=ns, exposures_per_band=epb,
                           shapes=[(side, side)] * sum(epb), n_psf=npsf, psf_sigma=(0.5, 4.0),
                           rot_deg=1.0, scale_frac=0.02, g_range=(0.8, 1.2), mask_frac=0.02,
                           flux_sigma=1.5)


@pytest.mark.skipif(not O.ref_available(), reason="reference CPU kernel not built")
@pytest.mark.parametrize("seed", [11, 12, 13])
def test_f32_oracle_bitexact_vs_reference_kernel(seed):
    P = synth.make_patch(_small_spec(4, [1, 2], 24), seed=seed)
    prop = P.proposal()
    a = O.oracle_evaluate(P, prop)
    b = O.ref_evaluate(P, prop)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.skipif(not O.ref_available(40), reason="MAXSOURCES=64 reference build missing")
def test_f32_oracle_bitexact_vs_reference_kernel_64_sources():
    P = synth.make_patch(_small_spec(40, [1], 16, npsf=1), seed=5)
    prop = P.proposal()
    a = O.oracle_evaluate(P, prop)
    b = O.ref_evaluate(P, prop)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_cutoff_changes_little():
    P, prop, d = load_golden("mini_3src_2band")
    a = O.oracle_evaluate(P, prop, precision="f64", cutoff=True)
    b = O.oracle_evaluate(P, prop, precision="f64", cutoff=False)
    np.testing.assert_allclose(a[0], b[0], rtol=1e-6)


def test_residual_output_matches_model():
    P, prop, d = load_golden("single_seed1")
    chi2, dchi2, res = O.oracle_evaluate(P, prop, residual=True)
    # chi2 recomputed from the residual with the kernel's offset form
    rie = res * P.ierr
    die = P.data * P.ierr
    c = np.sum((rie.astype(np.float64) - die) * (rie.astype(np.float64) + die))
    np.testing.assert_allclose(c, chi2[0], rtol=1e-12)
