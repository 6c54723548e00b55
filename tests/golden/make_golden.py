"""Generate the golden vectors in tests/golden/*.npz.

Run with the reference checkout named by --ref (or the FPHO_REFERENCE
environment variable) after ``make -C oracle all ref``:

    python tests/golden/make_golden.py --ref <reference checkout>

For each small seeded synthetic patch (forcepho_b200.synth) it stores the
packed patch arrays, the packed proposal and
  * ref_chi2, ref_dchi2 -- the reference's own CPU kernel
    (forcepho/src/compute_gaussians_kernel.cc, built by oracle/Makefile from its
    sources) through its pybind11 entry point EvaluateProposal(band, patch, proposal);
  * slow_chi2, slow_dchi2 -- the reference's FP64 python path
    (forcepho/slow/gaussmodel.py: _convert_to_gaussians, _get_gaussian_gradients,
    compute_gig), which has no exp-argument cutoff: chi2 in the kernels' offset
    form sum((r ie)^2 - (d ie)^2) and dchi2 = sum_p -2 r ie^2 dmodel/dtheta.
The reference tree is only read here; the fixtures are what travels.
"""

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from forcepho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

ARRAYS = ["data", "ierr", "xpix", "ypix", "exposure_start", "exposure_N", "band_start",
          "band_N", "rad2", "D", "crpix", "crval", "CW", "G", "n_psf_per_source", "psfgauss",
          "psfgauss_start"]


def import_slow(ref):
    m = types.ModuleType("forcepho")
    m.__path__ = [os.path.join(ref, "forcepho")]
    m.source_dir = os.path.join(ref, "forcepho", "src")
    sys.modules["forcepho"] = m
    from forcepho.slow import gaussmodel
    return gaussmodel


def slow_evaluate(gm, patch, proposal):
    """FP64 chi2 (offset form) and dchi2 per band from the slow path."""
    nb, ns = patch.n_bands, patch.n_sources
    chi2 = np.zeros(nb)
    dchi2 = np.zeros((nb, ns, 7))
    rad2 = patch.rad2.astype(np.float64)
    for b in range(nb):
        npsf = int(patch.n_psf_per_source[b])
        for e in range(int(patch.band_start[b]), int(patch.band_start[b] + patch.band_N[b])):
            p0, n = int(patch.exposure_start[e]), int(patch.exposure_N[e])
            xs = patch.xpix[p0:p0 + n].astype(np.float64)
            ys = patch.ypix[p0:p0 + n].astype(np.float64)
            d = patch.data[p0:p0 + n].astype(np.float64)
            ie = patch.ierr[p0:p0 + n].astype(np.float64)
            # the kernels read the PSF rows of source 0 of the exposure for all sources
            rows = patch.psfgauss[int(patch.psfgauss_start[e]):int(patch.psfgauss_start[e]) + npsf]
            model = np.zeros(n)
            grads = []
            for s in range(ns):
                src = proposal[s]
                q, pa = float(src["q"]), float(src["pa"])
                D = patch.D[e, s].astype(np.float64)
                CW = patch.CW[e, s].astype(np.float64)
                G = float(patch.G[e])
                flux = float(src["fluxes"][b])
                R = gm.rotation_matrix(pa)
                S = gm.scale_matrix(q)
                T = gm.fast_dot_dot_2x2(D, R, S)
                dT_dq = gm.fast_dot_dot_2x2(D, R, gm.scale_matrix_deriv(q))
                dT_dpa = gm.fast_dot_dot_2x2(D, gm.rotation_matrix_deriv(pa), S)
                smean = np.dot(CW, np.array([src["ra"], src["dec"]], dtype=np.float64)
                               - patch.crval[e, s].astype(np.float64)) + patch.crpix[e, s]
                gig = gm.GaussianImageGalaxy(npsf, 1)
                gig.gaussians = []
                for row in rows:
                    k = int(row["sersic_bin"])
                    scovar = rad2[k] * np.eye(2)[None]
                    pc = np.array([[[row["Cxx"], row["Cxy"]], [row["Cxy"], row["Cyy"]]]],
                                  dtype=np.float64)
                    samps = np.array([src["mixture_amplitudes"][k]], dtype=np.float64)
                    pamps = np.array([row["amp"]], dtype=np.float64)
                    pmeans = np.array([[row["xcen"], row["ycen"]]], dtype=np.float64)
                    scov_im = gm.fast_matmul_matmul_2x2(T, scovar, T.T)
                    g = gm._convert_to_gaussians(1, 1, scov_im, pc, smean, samps, pmeans, pamps,
                                                 flux * G)[0]
                    der = gm._get_gaussian_gradients(
                        1, 1, scovar, pc, samps, pamps, flux, G, T, dT_dq, dT_dpa,
                        np.array([src["damplitude_dnsersic"][k]], dtype=np.float64),
                        np.array([src["damplitude_drh"][k]], dtype=np.float64), CW)
                    g.derivs = der[0, 0]
                    gig.gaussians.append(g)
                im, gr = gm.compute_gig(gig, xs, ys, compute_deriv=True)
                model += im
                grads.append(gr)
            r = d - model
            chi2[b] += np.sum((r * ie) ** 2 - (d * ie) ** 2)
            w = -2.0 * r * ie * ie
            for s in range(ns):
                dchi2[b, s] += grads[s] @ w
    return chi2, dchi2


def cases():
    """(name, patch) of the committed fixtures."""
    out = [("single_seed1", synth.make_workload("single", seed=1)),
           ("single_seed7", synth.make_workload("single", seed=7))]
    spec = synth.PatchSpec(n_sources=3, exposures_per_band=[2, 1], shapes=[(40, 40), (37, 45),
                                                                           (40, 40)],
                           n_psf=2, psf_sigma=(0.5, 4.0), rot_deg=1.0, scale_frac=0.02,
                           g_range=(0.8, 1.2), mask_frac=0.02, flux_sigma=1.5)
    out.append(("mini_3src_2band", synth.make_patch(spec, seed=3)))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("FPHO_REFERENCE"))
    a = ap.parse_args()
    if not a.ref:
        ap.error("name the reference checkout with --ref or FPHO_REFERENCE")
    O.build(ref=a.ref)
    gm = import_slow(a.ref)
    for name, P in cases():
        prop = P.proposal()
        rc, rd = O.ref_evaluate(P, prop)
        sc, sd = slow_evaluate(gm, P, prop)
        arrs = {k: getattr(P, k) for k in ARRAYS}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), n_sources=P.n_sources,
                            n_radii=P.n_radii, proposal=prop, ref_chi2=rc, ref_dchi2=rd,
                            slow_chi2=sc, slow_dchi2=sd, **arrs)
        print(name, "ref chi2", rc, "slow chi2", sc)


if __name__ == "__main__":
    main()
