"""Python access to the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker; the forcepho_b200 product never imports it.

  oracle_evaluate(patch, proposal, precision="f32" | "f64", cutoff=True)
      the C restatement in oracle/fpho_oracle.c of the reference CPU kernel
      (forcepho/src/compute_gaussians_kernel.cc:227-315), band by band;
  ref_evaluate(patch, proposal)
      the reference's own CPU kernel, compiled from its sources by
      oracle/Makefile into oracle/_ref/ (the MAXSOURCES=64 build is used for
      patches with more than 30 sources).
"""

import ctypes
import glob
import importlib.util
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


def build(ref=None):
    """make -C oracle (and the reference build when its sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all", f"PY={sys.executable}"], check=True)
    src = ref if ref is not None else "/root/reference"
    if os.path.isdir(os.path.join(src, "forcepho", "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={src}", f"PY={sys.executable}"],
                       check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.fpo_evaluate_band_f32.argtypes = [ip, vp, vp, vp, vp, vp]
        L.fpo_evaluate_band_f32.restype = ip
        L.fpo_evaluate_band_f64.argtypes = [ip, vp, vp, ip, vp, vp, vp]
        L.fpo_evaluate_band_f64.restype = ip
        L.fpo_image_gaussians_f32.argtypes = [ip, ip, vp, vp, vp]
        L.fpo_image_gaussians_f32.restype = ip
        for n in ("fpo_sizeof_patch", "fpo_sizeof_source", "fpo_sizeof_psfgauss"):
            getattr(L, n).restype = ip
        _lib = L
    return _lib


def oracle_evaluate(patch, proposal, precision="f32", cutoff=True, residual=False, bands=None):
    """chi2 (n_bands,), dchi2 (n_bands, n_src, 7) [, residual (npix,)]."""
    L = lib()
    st = patch.host_struct()
    prop = np.ascontiguousarray(proposal)
    nb, ns = patch.n_bands, patch.n_sources
    bands = range(nb) if bands is None else bands
    chi2 = np.zeros(nb)
    if precision == "f32":
        dchi2 = np.zeros((nb, ns, 7), dtype=np.float32)
        res = np.zeros(patch.npix, dtype=np.float32) if residual else None
    else:
        dchi2 = np.zeros((nb, ns, 7), dtype=np.float64)
        res = np.zeros(patch.npix, dtype=np.float64) if residual else None
    for b in bands:
        c = ctypes.c_double(0.0)
        g = np.zeros(ns * 7, dtype=dchi2.dtype)
        rp = res.ctypes.data if res is not None else None
        if precision == "f32":
            rc = L.fpo_evaluate_band_f32(b, st.ctypes.data, prop.ctypes.data, ctypes.byref(c),
                                         g.ctypes.data, rp)
        else:
            rc = L.fpo_evaluate_band_f64(b, st.ctypes.data, prop.ctypes.data, int(bool(cutoff)),
                                         ctypes.byref(c), g.ctypes.data, rp)
        if rc != 0:
            raise MemoryError("oracle allocation failed")
        chi2[b] = c.value
        dchi2[b] = g.reshape(ns, 7)
    if residual:
        return chi2, dchi2, res
    return chi2, dchi2


def image_gaussians_f32(patch, proposal, band, exposure):
    """float32 array (n_sources * n_psf, 21) of the reference's ImageGaussians."""
    L = lib()
    st = patch.host_struct()
    prop = np.ascontiguousarray(proposal)
    n = patch.n_sources * int(patch.n_psf_per_source[band])
    out = np.zeros((n, 21), dtype=np.float32)
    L.fpo_image_gaussians_f32(band, exposure, st.ctypes.data, prop.ctypes.data, out.ctypes.data)
    return out


# ---------------------------------------------------------------- reference kernel
_ref_mods = {}


def _ref_module(ms64=False):
    key = "ms64" if ms64 else "std"
    if key not in _ref_mods:
        d = os.path.join(REF_DIR, "ms64") if ms64 else REF_DIR
        cands = glob.glob(os.path.join(d, "compute_gaussians_kernel*.so"))
        if not cands:
            _ref_mods[key] = None
        else:
            name = "compute_gaussians_kernel"
            spec = importlib.util.spec_from_file_location(name, cands[0])
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            _ref_mods[key] = mod
    return _ref_mods[key]


def ref_available(n_sources=1):
    return _ref_module(ms64=n_sources > 30) is not None


def ref_evaluate(patch, proposal, bands=None):
    """Run the reference CPU kernel band by band (as CPUProposer,
    forcepho/proposal.py:180-226).  Returns chi2 (n_bands,), dchi2
    (n_bands, n_src, 7) float32."""
    ns = patch.n_sources
    ms64 = ns > 30
    mod = _ref_module(ms64)
    if mod is None:
        raise RuntimeError("reference CPU kernel not built (make -C oracle ref)")
    maxsrc = 64 if ms64 else 30
    st = patch.host_struct()
    prop = np.ascontiguousarray(proposal)
    nb = patch.n_bands
    bands = range(nb) if bands is None else bands
    chi2 = np.zeros(nb)
    dchi2 = np.zeros((nb, ns, 7), dtype=np.float32)
    for b in bands:
        r = mod.EvaluateProposal(b, st.ctypes.data, prop.ctypes.data)
        chi2[b] = r.chi2
        dchi2[b] = np.asarray(r.dchi2_dp).reshape(maxsrc, 7)[:ns]
    return chi2, dchi2
