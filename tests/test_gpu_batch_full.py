"""Batched-path parity at full size: the 256 uneven patches the benchmark's
batched leg times (sources U{1..30}, bands U{1..8}, exposures per band
U{1..8}, 32-200 px per side; seed 3), evaluated in one batch through
PatchBatch.evaluate and through BatchPosterior.lnprob_and_grad, with 16 of
them -- the costliest, the 30-source patch with the most pixels, the
cheapest, and 13 spread over the cost order -- compared with the reference's
own CPU kernel (oracle/_ref) on the same proposals:

  * chi2 per band within 1e-6 relative;
  * gradients per component by the parity bar of test_gpu_parity.grad_ok
    (1e-5 relative, or the condition-scale allowance on ill-conditioned
    components against the exact sum over the reference's float Gaussians);
  * BatchPosterior: its device-built proposals are read back and given to
    the reference kernel; lnp per patch and d lnp / dz follow from the
    reference's chi2 and gradient through the bounded transform.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from test_gpu_parity import CHI2_RTOL, GRAD_RTOL, grad_ok

pytestmark = pytest.mark.gpu

SEED = 3             # the benchmark's batched-leg seed (its --seed 0 plus 3)
N_PATCHES = 256
N_CHECK = 16


@pytest.fixture(scope="module")
def pools():
    """Spawn pools for the reference kernel and the mixed oracle, started
    before the module's first GPU call."""
    cores = max(1, min(16, len(os.sched_getaffinity(0))))
    if not O.ref_available(1):
        pytest.skip("reference CPU kernel not built (oracle/_ref)")
    ref = O.ref_pool(1, cores)
    mixed = O.oracle_pool(cores)
    yield ref, mixed
    for p in (ref, mixed):
        p.close()
        p.join()


@pytest.fixture(scope="module")
def uneven(pools):
    from forcepho_b200 import synth
    patches = synth.make_workload("uneven", seed=SEED, render=synth.render_model_gpu,
                                  n_patches=N_PATCHES)
    for P in patches:
        P.return_residual = False
        P.send_to_device()
    cost = np.array([P.pairs_per_eval for P in patches])
    order = np.argsort(cost)
    pick = {int(order[-1]), int(order[0])}
    thirty = [i for i, P in enumerate(patches) if P.n_sources == max(q.n_sources for q in patches)]
    pick.add(max(thirty, key=lambda i: patches[i].npix))
    for j in np.linspace(1, len(order) - 2, N_CHECK).astype(int):
        if len(pick) >= N_CHECK:
            break
        pick.add(int(order[j]))
    yield patches, sorted(pick)
    for P in patches:
        P.free()


def check_grad_pooled(g, ref, P, prop, pool):
    """The per-component bar of test_gpu_parity.check_grad, with the mixed
    oracle run (in `pool`, band by band) only for bands where some component
    misses the plain 1e-5 bar.  Returns the fraction within 1e-5."""
    g = np.asarray(g, np.float64)
    ref = np.asarray(ref, np.float64)
    plain = np.abs(g - ref) <= GRAD_RTOL * np.abs(ref)
    bad_bands = [b for b in range(P.n_bands) if not plain[b].all()]
    if bad_bands:
        res = O.mixed_abs_many(P, [(prop, b) for b in bad_bands], pool)
        mixed = np.stack([r[2] for r in res])
        scale = np.stack([r[3] for r in res])
        rscale = np.stack([r[5] for r in res])
        ok = grad_ok(g[bad_bands], ref[bad_bands], mixed, scale, rscale)
        assert np.all(ok), (f"{(~ok).sum()} components: gpu {g[bad_bands][~ok]}, ref "
                            f"{ref[bad_bands][~ok]}, mixed {mixed[~ok]}")
    return float(plain.mean())


def test_uneven_batch_vs_reference(uneven, pools):
    """PatchBatch.evaluate over all 256 patches; 16 compared with the reference."""
    from forcepho_b200.batch import PatchBatch
    patches, pick = uneven
    ref_pool, mixed_pool = pools
    batch = PatchBatch(patches)
    props = [P.proposal() for P in patches]
    chi2_b, dchi2_b = batch.evaluate(props)
    assert batch.error_word() == 0
    fracs = []
    for i in pick:
        P, q = patches[i], props[i]
        c_ref, g_ref = O.ref_evaluate(P, q, pool=ref_pool)
        np.testing.assert_allclose(chi2_b[i], c_ref, rtol=CHI2_RTOL)
        fracs.append(check_grad_pooled(dchi2_b[i], g_ref, P, q, mixed_pool))
    sizes = [(patches[i].n_sources, patches[i].n_exp, patches[i].npix) for i in pick]
    print("checked (sources, exposures, pixels):", sizes)
    print("fraction of components within 1e-5 of the reference:", np.mean(fracs))
    batch.free()


def test_uneven_batch_posterior_vs_reference(uneven, pools):
    """BatchPosterior.lnprob_and_grad over all 256 patches at a perturbed
    position; per checked patch, lnp and d lnp / dz against the reference
    kernel evaluated on the proposals the device built."""
    import torch
    from forcepho_b200.autograd import BatchPosterior, default_bounds
    from forcepho_b200.batch import PatchBatch
    from forcepho_b200.model import BoundedTransform, stack_band_gradients
    from forcepho_b200.proposal import source_struct_dtype
    patches, pick = uneven
    ref_pool, mixed_pool = pools
    batch = PatchBatch(patches)
    lows, highs = zip(*[default_bounds(P.params, P.n_bands) for P in patches])
    bp = BatchPosterior(batch, lows, highs)
    rng = np.random.default_rng(17)
    q0 = np.concatenate([P.params.reshape(-1) for P in patches])
    lo, hi = np.concatenate(lows), np.concatenate(highs)
    q = np.clip(q0 + 0.01 * (hi - lo) * rng.standard_normal(q0.shape), lo + 1e-3 * (hi - lo),
                hi - 1e-3 * (hi - lo))
    z = bp.inverse_transform(torch.as_tensor(q, device="cuda"))
    lnp, g = bp.lnprob_and_grad(z)
    lnp_k = bp.lnp_per_patch(z).cpu().numpy()
    torch.cuda.synchronize()
    assert batch.error_word() == 0
    g = g.cpu().numpy()
    zc = z.cpu().numpy()
    assert float(lnp) == pytest.approx(float(lnp_k.sum()), rel=1e-12)
    props = np.frombuffer(bp.prop.cpu().numpy().tobytes(), dtype=source_struct_dtype)
    chi2_dev, dchi2_dev = batch.split_outputs(bp.chi2.cpu().numpy(), bp.dchi2.cpu().numpy())
    ns = np.array([P.n_sources for P in patches])
    nb = np.array([P.n_bands for P in patches])
    src_off = np.concatenate([[0], np.cumsum(ns)])
    par_off = np.concatenate([[0], np.cumsum(ns * (nb + 6))])
    for i in pick:
        P = patches[i]
        prop = np.ascontiguousarray(props[src_off[i]:src_off[i + 1]])
        c_ref, g_ref = O.ref_evaluate(P, prop, pool=ref_pool)
        np.testing.assert_allclose(chi2_dev[i], c_ref, rtol=CHI2_RTOL)
        check_grad_pooled(dchi2_dev[i], g_ref, P, prop, mixed_pool)
        # lnp and d lnp/dz of this patch from the reference's chi2 and gradient
        sl = slice(par_off[i], par_off[i + 1])
        T = BoundedTransform(lows[i], highs[i])
        want_lnp = -0.5 * c_ref.sum() + T.lndetjac(zc[sl])
        assert lnp_k[i] == pytest.approx(want_lnp, rel=CHI2_RTOL)
        # the device's stacking and chain rule, on the device's own gradient
        gz_dev = -0.5 * stack_band_gradients(dchi2_dev[i], P.n_bands) * T.jacobian(zc[sl]) + \
            T.lndetjac_grad(zc[sl])
        np.testing.assert_allclose(g[sl], gz_dev, rtol=1e-9, atol=1e-9 * np.abs(gz_dev).max())
    batch.free()
