"""Linear flux solve on top of the design matrix.

Mirrors forcepho/fitting.py:573-627: :func:`optimize_one_band` (weighted
least squares for one band: Xp = X w, yp = (y - fixedX) w, ATA = Xp Xp^T,
fluxes = solve(ATA, Xp yp)) and :func:`optimize_fluxes` (the maximum-
likelihood fluxes and flux precision matrices of the active sources,
conditional on their shapes, from ``patcher.design_matrix``).
:func:`optimize_fluxes_device` does the same without leaving the GPU: the
design matrix from one ``fpho_patch_design_matrix`` launch, the normal
equations as FP64 matrix products (cuBLAS through torch), the solves by
torch.linalg.
"""

import numpy as np

__all__ = ["optimize_one_band", "optimize_fluxes", "optimize_fluxes_device"]


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


def optimize_fluxes_device(patcher, active):
    """As :func:`optimize_fluxes`, computed on the GPU: returns (fluxes
    (n_bands, n_source), precisions (n_bands, n_source, n_source)) as float64
    CUDA tensors."""
    import torch
    scene = active if hasattr(active, "get_proposal") else patcher.set_scene(active)
    patcher.pack_meta(scene)
    patcher.replace_device_meta_ptrs()
    X = patcher.design_matrix_device(scene.get_proposal()).to(torch.float64)
    y = torch.as_tensor(patcher.retrieve_array("data"), device="cuda", dtype=torch.float64)
    w = torch.as_tensor(patcher.ierr, device="cuda", dtype=torch.float64)
    cuts = np.concatenate([[0], np.cumsum(patcher.band_N_pix)])
    fl, pr = [], []
    for b in range(patcher.n_bands):
        sl = slice(int(cuts[b]), int(cuts[b + 1]))
        Xp = X[:, sl] * w[sl]
        yp = y[sl] * w[sl]
        ata = Xp @ Xp.T
        fl.append(torch.linalg.solve(ata, Xp @ yp))
        pr.append(ata)
    return torch.stack(fl), torch.stack(pr)
