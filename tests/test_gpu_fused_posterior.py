"""GPU: the fused posterior launches against the unfused torch form.

DevicePosterior and BatchPosterior build the proposal through the bounded
transform in one launch (fpho_build_proposal_bounded) and form lnp and its
gradient in one launch (fpho_bounded_lnp_grad).  Their results must equal
the elementwise torch form (sigmoid, proposal build, stacking of the per-band
gradient) at the same z: lnp to 1e-12 relative, every gradient component to
1e-12 of the largest, on the 20-source patch, on uneven batches and at points
near the bounds; and a leapfrog trajectory captured in a CUDA graph through
the fused form must follow the unfused one.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(post, z):
    import torch
    lnp_f, g_f = post.lnprob_and_grad(z)
    lnp_f, g_f = float(lnp_f), g_f.clone()
    lnp_t, g_t = post._lnprob_and_grad_torch(z)
    torch.cuda.synchronize()
    lnp_t = float(lnp_t)
    assert np.isfinite(lnp_f)
    assert abs(lnp_f - lnp_t) <= 1e-12 * abs(lnp_t)
    scale = float(g_t.abs().max())
    assert float((g_f - g_t).abs().max()) <= 1e-12 * scale
    return lnp_f


def test_device_posterior_fused_matches_torch():
    import torch
    from forcepho_b200 import synth
    from forcepho_b200.autograd import DevicePosterior, default_bounds
    P = synth.make_workload("field20", seed=0, render=synth.render_model_gpu)
    P.return_residual = False
    P.send_to_device()
    lo, hi = default_bounds(P.params, P.n_bands)
    post = DevicePosterior(P, lo, hi)
    z0 = post.inverse_transform(P.params.reshape(-1))
    rng = np.random.default_rng(2)
    for scale in (0.0, 1e-2, 0.3):
        z = z0 + torch.as_tensor(scale * rng.standard_normal(post.ndim), device="cuda")
        _check(post, z)
    # near the bounds: s close to 0 and 1
    z = z0.clone()
    z[::5] = 12.0
    z[1::5] = -12.0
    _check(post, z)
    P.free()


def test_batch_posterior_fused_matches_torch():
    import torch
    from forcepho_b200 import synth
    from forcepho_b200.autograd import BatchPosterior, default_bounds
    from forcepho_b200.batch import PatchBatch
    patches = synth.make_workload("uneven", seed=3, render=synth.render_model_gpu, n_patches=6)
    for p in patches:
        p.return_residual = False
        p.send_to_device()
    bounds = [default_bounds(p.params, p.n_bands) for p in patches]
    batch = PatchBatch(patches)
    post = BatchPosterior(batch, [b[0] for b in bounds], [b[1] for b in bounds])
    z0 = post.inverse_transform(np.concatenate([p.params.reshape(-1) for p in patches]))
    rng = np.random.default_rng(5)
    for scale in (0.0, 0.1):
        z = z0 + torch.as_tensor(scale * rng.standard_normal(post.ndim), device="cuda")
        _check(post, z)
    batch.free()
    for p in patches:
        p.free()


def test_leapfrog_fused_follows_unfused():
    import torch
    from forcepho_b200 import synth
    from forcepho_b200.autograd import DevicePosterior, Leapfrog, default_bounds
    P = synth.make_workload("single", seed=1, render=synth.render_model_gpu)
    P.send_to_device()
    lo, hi = default_bounds(P.params, P.n_bands)
    post = DevicePosterior(P, lo, hi)
    z0 = post.inverse_transform(P.params.reshape(-1))
    p0 = torch.as_tensor(np.random.default_rng(7).standard_normal(post.ndim), device="cuda")

    class Unfused:
        ndim = post.ndim

        def lnprob_and_grad(self, z):
            return post._lnprob_and_grad_torch(z)

    out = []
    for target in (post, Unfused()):
        lf = Leapfrog(target, eps=1e-3, steps_per_graph=10)
        lf.set_state(z0, p0)
        lf.run(50)
        torch.cuda.synchronize()
        out.append((lf.z.clone(), float(lf.hamiltonian())))
        del lf
    (za, ha), (zb, hb) = out
    assert float((za - zb).abs().max()) <= 1e-9 * float(zb.abs().max())
    assert abs(ha - hb) <= 1e-9 * abs(hb)
    P.free()
