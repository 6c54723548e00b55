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
