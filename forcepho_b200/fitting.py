"""Linear flux solve on top of the design matrix.

Mirrors forcepho/fitting.py:573-627: :func:`optimize_one_band` (weighted
least squares for one band: Xp = X w, yp = (y - fixedX) w, ATA = Xp Xp^T,
fluxes = solve(ATA, Xp yp)) and :func:`optimize_fluxes` (the maximum-
likelihood fluxes and flux precision matrices of the active sources,
conditional on their shapes, from ``patcher.design_matrix``).
:func:`optimize_fluxes_device` does the same without leaving the GPU and
without forming the design matrix: ``fpho_patch_optimize_fluxes`` builds each
tile's unit-flux models in shared memory, reduces the FP64 normal equations
per band in a fixed order and solves them by Cholesky factorisation, on the
patch's device data (after ``subtract_fixed``, the data less the fixed
sources).

:func:`run_hmc` and :func:`run_opt` keep the call shape and the result
fields of forcepho's ``run_lmc`` and ``run_opt`` (fitting.py:255-342,
415-454).  ``run_hmc`` samples with :class:`forcepho_b200.sampling.MultiChainHMC`
on the GPU (static-length HMC with a jittered step size, one CUDA graph per
iteration, any number of chains in one batched launch) instead of
littlemcmc's NUTS on the host; ``run_opt`` is the same BFGS minimisation of
the negative log posterior with scipy.
"""

import numpy as np

__all__ = ["optimize_one_band", "optimize_fluxes", "optimize_fluxes_device", "Result",
           "run_hmc", "run_opt"]


def optimize_one_band(X, w, y, fixedX=0):
    """Maximum-likelihood fluxes (n_source, 1) and precision matrix
    (n_source, n_source) for one band (X: (n_source, n_pix), w = ierr)."""
    Xp = X * w
    yp = (y - fixedX) * w
    ATA = np.dot(Xp, Xp.T)
    Xyp = np.dot(Xp, yp[:, None])
    flux = np.linalg.solve(ATA, Xyp)
    return flux, ATA


def optimize_fluxes(patcher, active, return_all=False):
    """Fluxes (list over bands of (n_source,)) and precisions (list of
    (n_source, n_source)); the design matrix comes from the device."""
    from numpy.linalg import LinAlgError
    fluxes, precisions = [], []
    Xes, ys = patcher.design_matrix(active)
    ws = patcher.split_band("ierr")
    for i, (w, X, y) in enumerate(zip(ws, Xes, ys)):
        try:
            flux, precision = optimize_one_band(X.astype(np.float64), w.astype(np.float64),
                                                y.astype(np.float64))
            fluxes.append(np.atleast_1d(np.squeeze(flux)))
            precisions.append(precision)
        except LinAlgError as e:
            return i, e, Xes, ys, ws
    if return_all:
        return fluxes, precisions, Xes, ys, ws
    return fluxes, precisions


def optimize_fluxes_device(patcher, active, stream=None, return_status=False):
    """As :func:`optimize_fluxes`, computed on the GPU in one call of
    ``fpho_patch_optimize_fluxes``: returns (fluxes (n_bands, n_source),
    precisions (n_bands, n_source, n_source)) as float64 CUDA tensors, and
    with `return_status` an int32 tensor (n_bands,) that is 1 where a band's
    precision matrix is not positive definite (its fluxes are NaN).  Nothing
    is synchronized or copied to the host."""
    import torch
    from . import _lib
    scene = active if hasattr(active, "get_proposal") else patcher.set_scene(active)
    patcher.pack_meta(scene)
    patcher.replace_device_meta_ptrs()
    prop = np.ascontiguousarray(scene.get_proposal())
    ns, nb = len(prop), int(patcher.n_bands)
    dprop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    flux = torch.empty((nb, ns), dtype=torch.float64, device="cuda")
    prec = torch.empty((nb, ns, ns), dtype=torch.float64, device="cuda")
    status = torch.zeros(nb, dtype=torch.int32, device="cuda")
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    _lib.call("fpho_patch_optimize_fluxes", patcher.device_patch.handle, dprop.data_ptr(), ns,
              flux.data_ptr(), prec.data_ptr(), status.data_ptr(), s)
    if return_status:
        return flux, prec, status
    return flux, prec


class Result:
    """The fields forcepho's run_lmc / run_opt fill (fitting.py:318-342,
    437-454): ndim, starting_position, chain, n_call, wall_time, and what
    each sampler adds (lnp, fun, jac, message; accept, step_size)."""

    def __init__(self, filename=None, **kw):
        self.__dict__.update(kw)
        if filename is not None:
            self.read_from_h5(filename)

    def dump_to_h5(self, filename, verbose=False):
        """Save the attributes to an HDF5 file as forcepho's Result does
        (fitting.py:186-207): arrays as datasets, other values as attributes
        of the root group; returns messages for values that cannot be stored."""
        import os
        from . import h5lite
        datasets, attrs, msgs = {}, {}, []
        for name, value in vars(self).items():
            if isinstance(value, np.ndarray) and value.dtype != object:
                datasets[name] = value
            elif isinstance(value, (str, bytes, bool, int, float, np.generic)):
                attrs[name] = value
            else:
                msgs.append(f"could not save {name} with value {value!r} to {filename}")
        if verbose:
            for m in msgs:
                print(m)
        d = os.path.dirname(filename)
        if d:
            os.makedirs(d, exist_ok=True)
        h5lite.write(filename, datasets, {"/": attrs})
        return msgs

    def read_from_h5(self, filename):
        """Read the datasets and root attributes of an HDF5 file (written by
        :meth:`dump_to_h5` or by forcepho) into attributes."""
        from . import h5lite
        with h5lite.File(filename) as f:
            for k in f.keys():
                node = f[k]
                if not isinstance(node, h5lite.Group):
                    setattr(self, k, node[...] if not node.shape else np.array(node[:]))
            for k, v in f.attrs.items():
                setattr(self, k, v)
        return self


def run_hmc(model, q, n_draws, warmup=(10,), n_chains=1, n_leapfrog=10, step_size=0.05,
            target_accept=0.75, jitter=0.2, random_seed=0xDEADBEEF, z_cov=None, full=False,
            adapt=False):
    """HMC on the GPU with the call shape of forcepho's ``run_lmc``.

    Parameters
    ----------
    model : forcepho_b200.autograd.DevicePosterior (one patch; chains are
        device copies of it) or BatchPosterior (one chain per patch), or any
        object with the BatchPosterior sampling interface
    q : starting position in the constrained space, one chain's (broadcast
        to every chain) or all chains' concatenated
    n_draws : samples kept per chain
    warmup : lengths of the tuning rounds; in each the step size adapts
        every iteration by dual averaging towards `target_accept` (the
        chains' mean acceptance probability), and the averaged value is kept
        at the end of the round
    n_chains : chains of a DevicePosterior model (ignored for a batch)
    z_cov : the inverse mass matrix in the unconstrained coordinates z, as
        the reference's ``z_cov``: a vector of variances (one chain's, or all
        chains'), or with `full` a (d, d) covariance for every chain;
        default the identity
    full : a dense inverse mass matrix per chain (chains of equal size)
        instead of a diagonal
    adapt : after each warm-up round of at least 10 iterations, set the
        inverse mass matrix to the (co)variance of that round's samples,
        pooled over the chains when they are copies of one patch,
        regularised towards the identity (as the reference's adapting
        potential does, forcepho/fitting.py:370-413)

    Returns
    -------
    result : Result with ``chain`` of shape (n_draws, ndim) for one chain or
        (n_chains, n_draws, ndim), in the constrained space, ``n_call`` (one
        per chain per leapfrog step), ``wall_time``, ``accept`` (per chain,
        production iterations), ``step_size``
    sampler : the MultiChainHMC (``scale`` / ``chol``: the inverse-mass factors)
    """
    import time
    import torch
    from .autograd import BatchPosterior, DevicePosterior
    from .sampling import MultiChainHMC, chain_posterior, estimate_mass
    pooled = False
    if isinstance(model, DevicePosterior):
        lo = model.tr.lower.cpu().numpy()
        hi = model.tr.upper.cpu().numpy()
        post = chain_posterior(model.ev.patch, int(n_chains), lo, hi)
        pooled = True
    elif isinstance(model, BatchPosterior) or all(
            hasattr(model, a) for a in ("lnp_per_patch", "n_patches", "par_pad", "par_patch")):
        post, n_chains = model, model.n_patches
        pooled = getattr(model, "copies", None) is not None
    else:
        raise TypeError("model must be a DevicePosterior or a BatchPosterior")
    q = np.asarray(q, dtype=np.float64).reshape(-1)
    if q.size * n_chains == post.ndim:
        q = np.tile(q, n_chains)
    if q.size != post.ndim:
        raise ValueError(f"q has {q.size} entries; the chains need {post.ndim}")
    device = getattr(post, "device", "cuda")
    z0 = post.inverse_transform(torch.as_tensor(q, device=device))
    n_buf = max([int(n_draws)] + [int(w) for w in warmup])
    hmc = MultiChainHMC(post, step_size, n_leapfrog, n_samples=n_buf,
                        seed=int(random_seed) & 0x7FFFFFFF, jitter=jitter, full=full,
                        device=device)
    d = post.ndim // n_chains
    if z_cov is not None:
        zc = torch.as_tensor(np.asarray(z_cov, dtype=np.float64), device=device)
        if full:
            hmc.set_mass(chol=torch.linalg.cholesky(zc.reshape(d, d)))
        else:
            zc = zc.reshape(-1)
            hmc.set_mass(scale=(zc.repeat(n_chains) if zc.numel() == d else zc).sqrt())
    hmc.set_state(z0)
    t0 = time.time()
    for w in warmup:
        hmc.n_accept.zero_()
        hmc.slot.zero_()
        hmc.start_adaptation(target_accept)
        hmc.run(int(w))
        hmc.stop_adaptation()
        if adapt and int(w) >= 10:
            est = estimate_mass(hmc.samples[:int(w)], n_chains, full=full, pooled=pooled)
            # the step size is in whitened units: rescale it by the change of
            # the typical inverse-mass scale so the next round starts comparably
            old = hmc.chol.diagonal(dim1=1, dim2=2) if full else hmc.scale
            new = est.diagonal(dim1=1, dim2=2) if full else est
            hmc.set_eps(hmc.eps * float(torch.exp(torch.log(old).mean() -
                                                  torch.log(new).mean())))
            if full:
                hmc.set_mass(chol=est)
            else:
                hmc.set_mass(scale=est)
    hmc.n_accept.zero_()
    hmc.slot.zero_()
    hmc.run(int(n_draws))
    if hmc.device.type == "cuda":
        torch.cuda.synchronize()
    wall = time.time() - t0
    zs = hmc.samples[:int(n_draws)]  # the ring buffer started at slot 0 for the draws
    qs = post.transform(zs).cpu().numpy().reshape(int(n_draws), n_chains, -1)
    chain = qs.transpose(1, 0, 2)
    return Result(ndim=chain.shape[-1], starting_position=q.copy(),
                  chain=chain[0] if n_chains == 1 else chain,
                  n_call=int(n_chains * (sum(int(w) for w in warmup) + int(n_draws)) *
                             n_leapfrog),
                  wall_time=wall, accept=hmc.acceptance(int(n_draws)),
                  step_size=hmc.eps), hmc


def run_opt(model, q, jac=True, callback=None, **extras):
    """BFGS minimisation of ``model.nll`` with scipy, as forcepho's run_opt:
    start from the unconstrained image of `q`, return the optimum in the
    constrained space (``chain`` of shape (1, ndim)), lnp = -fun/2."""
    import time
    from scipy.optimize import minimize
    start = model.transform.inverse_transform(q) if model.transform is not None \
        else np.array(q, dtype=np.float64)
    t0 = time.time()
    if jac:
        res = minimize(model.nll, start.copy(), jac=True, method="BFGS", options=dict(extras),
                       callback=callback)
    else:
        res = minimize(model.nll_nograd, start.copy(), jac=None, method="BFGS",
                       options=dict(extras), callback=callback)
    chain = np.atleast_2d(res.x)
    if model.transform is not None:
        chain = model.transform.transform(chain)
    return Result(ndim=len(q), starting_position=np.array(q, dtype=np.float64).copy(),
                  chain=chain, lnp=-0.5 * res.fun, wall_time=time.time() - t0, fun=res.fun,
                  jac=res.jac, message=res.message), res
