"""The batched persistent evaluation against per-patch evaluation (same tile
shape, same reduction order: results must be bitwise equal) and against the
oracle; CUDA-graph replay of the batched evaluation."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def small_batch(n=6, seed=3):
    from forcepho_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        spec = synth.workload_spec("uneven", rng)
        spec.shapes = [(s[0] // 3 + 16, s[1] // 3 + 16) for s in spec.shapes]
        spec.n_sources = min(spec.n_sources, 8)
        out.append(synth.make_patch(spec, seed=int(rng.integers(1 << 30))))
    return out


def test_batch_matches_per_patch_bitwise():
    from forcepho_b200.batch import PatchBatch
    from forcepho_b200.proposal import GPUProposer
    patches = small_batch()
    for P in patches:
        P.return_residual = False
        P.send_to_device()
    batch = PatchBatch(patches)
    props = [P.proposal() for P in patches]
    chi2_b, dchi2_b = batch.evaluate(props)
    pr = GPUProposer()
    for P, q, cb, gb in zip(patches, props, chi2_b, dchi2_b):
        c, g = pr.evaluate_proposal(q, patch=P)
        assert np.array_equal(c, cb)
        assert np.array_equal(g, gb)
    # against the oracle
    for P, q, cb in zip(patches[:3], props[:3], chi2_b[:3]):
        c64, _ = O.oracle_evaluate(P, q, precision="f64")
        np.testing.assert_allclose(cb, c64, rtol=1e-6)
    batch.free()
    for P in patches:
        P.free()


def test_batch_graph_replay():
    import torch
    from forcepho_b200.batch import PatchBatch
    patches = small_batch(4, seed=5)
    for P in patches:
        P.return_residual = False
        P.send_to_device()
    batch = PatchBatch(patches)
    dprop, chi2, dchi2 = batch.device_buffers()
    batch.evaluate_device(dprop, chi2, dchi2)
    torch.cuda.synchronize()
    ref_c, ref_g = chi2.clone(), dchi2.clone()
    chi2.zero_()
    dchi2.zero_()
    g = batch.capture_graph(dprop, chi2, dchi2)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    assert torch.equal(chi2, ref_c) and torch.equal(dchi2, ref_g)
    del g
    batch.free()
    for P in patches:
        P.free()


def test_every_batch_candidate_matches_oracle():
    """Every configuration the batch autotuner can pick (tile variant with a
    batched kernel, stage size, persistent-grid cap) gives chi2 and gradients
    of every patch of a small uneven batch within the parity bars of the
    reference CPU kernel (restated by the oracle), with the per-component
    gradient bar of test_gpu_parity.grad_ok."""
    from forcepho_b200.autotune import batch_candidates, time_batch
    from forcepho_b200.batch import PatchBatch
    from test_gpu_parity import CHI2_RTOL, grad_ok
    patches = small_batch(5, seed=11)
    for P in patches:
        P.return_residual = False
        P.send_to_device()
    props = [P.proposal() for P in patches]
    refs = []
    for P, q in zip(patches, props):
        c, g = O.oracle_evaluate(P, q, precision="f32")
        _, mixed, scale, _, rscale = O.oracle_mixed_abs(P, q, terms=True)
        refs.append((c, g, mixed, scale, rscale))
    cands = batch_candidates()
    assert len({c[0] for c in cands}) >= 3
    for v, lc, ctas in cands:
        b = PatchBatch(patches, live_cap=lc, variant=v, ctas_per_sm=ctas)
        assert b.config == {"variant": v, "live_cap": lc, "ctas_per_sm": ctas}
        chi2_b, dchi2_b = b.evaluate(props)
        assert b.error_word() == 0
        for (c, g, mixed, scale, rscale), cb, gb in zip(refs, chi2_b, dchi2_b):
            np.testing.assert_allclose(cb, c, rtol=CHI2_RTOL)
            ok = grad_ok(gb, g, mixed, scale, rscale)
            assert np.all(ok), ((v, lc, ctas), int((~ok).sum()))
        b.free()
    # the timing used by the tuner runs on the same batch
    assert time_batch(patches, cands[0][0], cands[0][1], cands[0][2], reps=2) > 0
    for P in patches:
        P.free()
