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
    """make -C oracle, and the reference build when a reference checkout is
    given (`ref`, else the FPHO_REFERENCE environment variable) and holds
    its sources."""
    subprocess.run(["make", "-s", "-C", HERE, "all", f"PY={sys.executable}"], check=True)
    src = ref if ref is not None else os.environ.get("FPHO_REFERENCE", "")
    if src and os.path.isdir(os.path.join(src, "forcepho", "src")):
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
        L.fpo_evaluate_band_mixed.argtypes = [ip, vp, vp, ip, vp, vp, vp]
        L.fpo_evaluate_band_mixed.restype = ip
        L.fpo_image_gaussians_f32.argtypes = [ip, ip, vp, vp, vp]
        L.fpo_image_gaussians_f32.restype = ip
        for n in ("fpo_sizeof_patch", "fpo_sizeof_source", "fpo_sizeof_psfgauss"):
            getattr(L, n).restype = ip
        _lib = L
    return _lib


def oracle_evaluate(patch, proposal, precision="f32", cutoff=True, residual=False, bands=None):
    """chi2 (n_bands,), dchi2 (n_bands, n_src, 7) [, residual (npix,)].

    precision: "f32" (the reference CPU kernel restated, bit-identical),
    "f64" (everything in double), "mixed" (the reference's float image
    Gaussians, then double per-pixel math and accumulation)."""
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
            fn = L.fpo_evaluate_band_f64 if precision == "f64" else L.fpo_evaluate_band_mixed
            rc = fn(b, st.ctypes.data, prop.ctypes.data, int(bool(cutoff)), ctypes.byref(c),
                    g.ctypes.data, rp)
        if rc != 0:
            raise MemoryError("oracle allocation failed")
        chi2[b] = c.value
        dchi2[b] = g.reshape(ns, 7)
    if residual:
        return chi2, dchi2, res
    return chi2, dchi2


def oracle_f32_dsum(patch, proposal):
    """chi2 (n_bands,) and dchi2 (n_bands, n_src, 7) float64: the reference
    CPU kernel's own float per-pixel gradient terms (bit-identical to its
    arithmetic) accumulated in double instead of its running float sums
    (see fpo_evaluate_band_f32_dsum)."""
    L = lib()
    if not hasattr(L, "_dsum_bound"):
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.fpo_evaluate_band_f32_dsum.argtypes = [ip, vp, vp, vp, vp]
        L.fpo_evaluate_band_f32_dsum.restype = ip
        L._dsum_bound = True
    st = patch.host_struct()
    prop = np.ascontiguousarray(proposal)
    nb, ns = patch.n_bands, patch.n_sources
    chi2 = np.zeros(nb)
    dchi2 = np.zeros((nb, ns, 7))
    for b in range(nb):
        c = ctypes.c_double(0.0)
        g = np.zeros(ns * 7)
        if L.fpo_evaluate_band_f32_dsum(b, st.ctypes.data, prop.ctypes.data, ctypes.byref(c),
                                        g.ctypes.data) != 0:
            raise MemoryError("oracle allocation failed")
        chi2[b], dchi2[b] = c.value, g.reshape(ns, 7)
    return chi2, dchi2


def _worker_f32_dsum(payload, proposal, band):
    """(band, chi2, dchi2 (n_src, 7)) of oracle_f32_dsum for one band, in a
    worker process."""
    L = lib()
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.fpo_evaluate_band_f32_dsum.argtypes = [ip, vp, vp, vp, vp]
    L.fpo_evaluate_band_f32_dsum.restype = ip
    arrays, ns, nr = _resolve(payload)
    st = _struct_from_arrays(arrays, ns, nr)
    prop = np.ascontiguousarray(proposal)
    c = ctypes.c_double(0.0)
    g = np.zeros(ns * 7)
    if L.fpo_evaluate_band_f32_dsum(band, st.ctypes.data, prop.ctypes.data, ctypes.byref(c),
                                    g.ctypes.data) != 0:
        raise MemoryError("oracle allocation failed")
    return band, c.value, g.reshape(ns, 7)


def _worker_f32_res(payload, proposal, band):
    """(band, chi2, dchi2 (n_src, 7) float32, first pixel, residual of the
    band's pixels) of the f32 oracle (the reference kernel restated) for one
    band, in a worker process."""
    L = lib()
    arrays, ns, nr = _resolve(payload)
    st = _struct_from_arrays(arrays, ns, nr)
    prop = np.ascontiguousarray(proposal)
    e0 = int(arrays["band_start"][band])
    e1 = e0 + int(arrays["band_N"][band])
    lo = int(arrays["exposure_start"][e0])
    hi = int(arrays["exposure_start"][e1 - 1] + arrays["exposure_N"][e1 - 1])
    res = np.zeros(hi, dtype=np.float32)
    c = ctypes.c_double(0.0)
    g = np.zeros(ns * 7, dtype=np.float32)
    if L.fpo_evaluate_band_f32(band, st.ctypes.data, prop.ctypes.data, ctypes.byref(c),
                               g.ctypes.data, res.ctypes.data) != 0:
        raise MemoryError("oracle allocation failed")
    return band, c.value, g.reshape(ns, 7), lo, res[lo:hi].copy()


def _worker_res_dexp(payload, proposal, band, rounded_trig=0):
    """(band, first pixel, residual of the band's pixels) of
    fpo_residual_band_f32_dexp, in a worker process."""
    L = lib()
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.fpo_residual_band_f32_dexp.argtypes = [ip, vp, vp, vp, ip]
    L.fpo_residual_band_f32_dexp.restype = ip
    arrays, ns, nr = _resolve(payload)
    st = _struct_from_arrays(arrays, ns, nr)
    prop = np.ascontiguousarray(proposal)
    e0 = int(arrays["band_start"][band])
    e1 = e0 + int(arrays["band_N"][band])
    lo = int(arrays["exposure_start"][e0])
    hi = int(arrays["exposure_start"][e1 - 1] + arrays["exposure_N"][e1 - 1])
    res = np.zeros(hi, dtype=np.float32)
    if L.fpo_residual_band_f32_dexp(band, st.ctypes.data, prop.ctypes.data, res.ctypes.data,
                                    int(rounded_trig)):
        raise MemoryError("oracle allocation failed")
    return band, lo, res[lo:hi].copy()


def residual_dexp_many(patch, proposal, pool, bands=None, payload=None, rounded_trig=False):
    """The reference CPU kernel's residual image with a correctly rounded
    float exp in place of the C library's expf (fpo_residual_band_f32_dexp),
    and with `rounded_trig` correctly rounded cos/sin of the position angle
    in place of cosf/sinf; bands spread over `pool`; NaN outside the bands
    evaluated."""
    payload = payload or _patch_payload(patch)
    bands = range(patch.n_bands) if bands is None else bands
    res = np.full(patch.npix, np.nan, dtype=np.float32)
    prop = np.ascontiguousarray(proposal)
    jobs = [(payload, prop, b, int(rounded_trig)) for b in bands]
    for b, lo, r in pool.starmap(_worker_res_dexp, jobs):
        res[lo:lo + len(r)] = r
    return res


def f32_residual_many(patch, proposal, pool, bands=None, payload=None):
    """The f32 oracle (bit-identical to the reference CPU kernel) with its
    residual image, bands spread over `pool`: chi2 (n_bands,), dchi2
    (n_bands, n_src, 7) float32, residual (npix,) float32 (NaN outside the
    bands evaluated)."""
    payload = payload or _patch_payload(patch)
    nb, ns = patch.n_bands, patch.n_sources
    bands = range(nb) if bands is None else bands
    chi2 = np.full(nb, np.nan)
    dchi2 = np.full((nb, ns, 7), np.nan, dtype=np.float32)
    res = np.full(patch.npix, np.nan, dtype=np.float32)
    prop = np.ascontiguousarray(proposal)
    for b, c, g, lo, r in pool.starmap(_worker_f32_res, [(payload, prop, b) for b in bands]):
        chi2[b], dchi2[b] = c, g
        res[lo:lo + len(r)] = r
    return chi2, dchi2, res


def f32_dsum_many(patch, proposal, pool, bands=None, payload=None):
    """oracle_f32_dsum with the bands spread over `pool` (see oracle_pool);
    bands not in `bands` are left zero."""
    payload = payload or _patch_payload(patch)
    nb, ns = patch.n_bands, patch.n_sources
    bands = range(nb) if bands is None else bands
    chi2 = np.zeros(nb)
    dchi2 = np.zeros((nb, ns, 7))
    prop = np.ascontiguousarray(proposal)
    for b, c, g in pool.starmap(_worker_f32_dsum, [(payload, prop, b) for b in bands]):
        chi2[b], dchi2[b] = c, g
    return chi2, dchi2


def oracle_mixed_abs(patch, proposal, terms=False):
    """Mixed-precision evaluation (the reference's float image Gaussians,
    double pixel math) returning chi2, dchi2 (n_bands, n_src, 7) and, per
    component, the sum over pixels of |per-pixel contribution|; with
    ``terms``, also the sum over pixels and Gaussians of |each term| and the
    residual-rounding scale (see fpo_evaluate_band_mixed_abs)."""
    L = lib()
    if not hasattr(L, "_mixed_abs_bound"):
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.fpo_evaluate_band_mixed_abs.argtypes = [ip, vp, vp, ip, vp, vp, vp, vp, vp]
        L.fpo_evaluate_band_mixed_abs.restype = ip
        L._mixed_abs_bound = True
    st = patch.host_struct()
    prop = np.ascontiguousarray(proposal)
    nb, ns = patch.n_bands, patch.n_sources
    chi2 = np.zeros(nb)
    dchi2 = np.zeros((nb, ns, 7))
    dabs = np.zeros((nb, ns, 7))
    dterm = np.zeros((nb, ns, 7))
    dres = np.zeros((nb, ns, 7))
    for b in range(nb):
        c = ctypes.c_double(0.0)
        g = np.zeros(ns * 7)
        a = np.zeros(ns * 7)
        t = np.zeros(ns * 7)
        rs = np.zeros(ns * 7)
        if L.fpo_evaluate_band_mixed_abs(b, st.ctypes.data, prop.ctypes.data, 1, ctypes.byref(c),
                                         g.ctypes.data, a.ctypes.data, t.ctypes.data,
                                         rs.ctypes.data) != 0:
            raise MemoryError("oracle allocation failed")
        chi2[b], dchi2[b], dabs[b] = c.value, g.reshape(ns, 7), a.reshape(ns, 7)
        dterm[b], dres[b] = t.reshape(ns, 7), rs.reshape(ns, 7)
    if terms:
        return chi2, dchi2, dabs, dterm, dres
    return chi2, dchi2, dabs


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
# The reference builds (MAXSOURCES 30 and 64) are two pybind11 modules with the
# same name and types; a process may load only one of them.  This process
# loads the 30-source build; the 64-source build (and multi-process CPU
# baselines) run in worker processes started with `spawn`.
_ref_mod = None
PATCH_ARRAYS = ["data", "ierr", "xpix", "ypix", "exposure_start", "exposure_N", "band_start",
                "band_N", "rad2", "D", "crpix", "crval", "CW", "G", "n_psf_per_source",
                "psfgauss", "psfgauss_start"]


def _ref_path(ms64):
    d = os.path.join(REF_DIR, "ms64") if ms64 else REF_DIR
    c = glob.glob(os.path.join(d, "compute_gaussians_kernel*.so"))
    return c[0] if c else None


def _load_ref(ms64):
    spec = importlib.util.spec_from_file_location("compute_gaussians_kernel", _ref_path(ms64))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def ref_available(n_sources=1):
    return _ref_path(n_sources > 30) is not None


# the reference's Patch struct (forcepho/src/patch.cc:23-99) as a numpy record
_PTR = np.uintp
_STRUCT = np.dtype([("data", _PTR), ("ierr", _PTR), ("xpix", _PTR), ("ypix", _PTR),
                    ("residual", _PTR), ("exposure_start", _PTR), ("exposure_N", _PTR),
                    ("band_start", _PTR), ("band_N", _PTR), ("n_sources", np.int32),
                    ("n_radii", np.int32), ("rad2", _PTR), ("D", _PTR), ("crpix", _PTR),
                    ("crval", _PTR), ("CW", _PTR), ("G", _PTR), ("n_psf_per_source", _PTR),
                    ("psfgauss", _PTR), ("psfgauss_start", _PTR)], align=True)


def _struct_from_arrays(arrays, n_sources, n_radii):
    st = np.zeros(1, dtype=_STRUCT)
    for k, v in arrays.items():
        st[k] = v.ctypes.data
    st["n_sources"], st["n_radii"] = n_sources, n_radii
    return st


def _patch_payload(patch):
    return ({k: np.ascontiguousarray(getattr(patch, k)) for k in PATCH_ARRAYS},
            int(patch.n_sources), int(patch.n_radii))


def patch_payload_file(patch, path):
    """Write the patch arrays to `path` (.npz) once, so that worker jobs can
    name the file instead of pickling the arrays with every job."""
    arrays, ns, nr = _patch_payload(patch)
    np.savez(path, n_sources=ns, n_radii=nr, **arrays)
    return path


_payload_cache = {}


def _resolve(payload):
    if not isinstance(payload, str):
        return payload
    if payload not in _payload_cache:
        d = np.load(payload)
        arrays = {k: np.ascontiguousarray(d[k]) for k in PATCH_ARRAYS}
        _payload_cache.clear()
        _payload_cache[payload] = (arrays, int(d["n_sources"]), int(d["n_radii"]))
    return _payload_cache[payload]


_worker = {}


def _worker_init(ms64, root):
    if root not in sys.path:
        sys.path.insert(0, root)
    _worker["mod"] = _load_ref(ms64)
    _worker["ms64"] = ms64


def _worker_eval(payload, proposal, band, reps=1):
    import time
    arrays, ns, nr = _resolve(payload)
    st = _struct_from_arrays(arrays, ns, nr)
    prop = np.ascontiguousarray(proposal)
    maxsrc = 64 if _worker["ms64"] else 30
    t0 = time.perf_counter()
    for _ in range(reps):
        r = _worker["mod"].EvaluateProposal(band, st.ctypes.data, prop.ctypes.data)
    dt = time.perf_counter() - t0
    return band, r.chi2, np.asarray(r.dchi2_dp).reshape(maxsrc, 7)[:ns].copy(), dt


def ref_pool(n_sources, processes):
    """A spawn pool of `processes` workers, each with the reference build
    suited to `n_sources` loaded."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    root = os.path.dirname(HERE)
    return ctx.Pool(processes, initializer=_worker_init, initargs=(n_sources > 30, root))


def ref_evaluate(patch, proposal, bands=None, pool=None):
    """Run the reference CPU kernel band by band (as CPUProposer,
    forcepho/proposal.py:180-226).  Returns chi2 (n_bands,), dchi2
    (n_bands, n_src, 7) float32.  Patches of more than 30 sources, or a
    given `pool`, run in worker processes."""
    global _ref_mod
    ns = patch.n_sources
    nb = patch.n_bands
    bands = list(range(nb)) if bands is None else list(bands)
    chi2 = np.zeros(nb)
    dchi2 = np.zeros((nb, ns, 7), dtype=np.float32)
    if pool is None and ns <= 30:
        if _ref_path(False) is None:
            raise RuntimeError("reference CPU kernel not built (make -C oracle ref)")
        if _ref_mod is None:
            _ref_mod = _load_ref(False)
        st = patch.host_struct()
        prop = np.ascontiguousarray(proposal)
        for b in bands:
            r = _ref_mod.EvaluateProposal(b, st.ctypes.data, prop.ctypes.data)
            chi2[b] = r.chi2
            dchi2[b] = np.asarray(r.dchi2_dp).reshape(30, 7)[:ns]
        return chi2, dchi2
    own = pool is None
    if own:
        if _ref_path(ns > 30) is None:
            raise RuntimeError("reference CPU kernel not built (make -C oracle ref)")
        pool = ref_pool(ns, 1)
    try:
        payload = _patch_payload(patch)
        prop = np.ascontiguousarray(proposal)
        res = pool.starmap(_worker_eval, [(payload, prop, b) for b in bands])
    finally:
        if own:
            pool.close()
            pool.join()
    for b, c, g, _ in res:
        chi2[b] = c
        dchi2[b] = g
    return chi2, dchi2


# ---------------------------------------------------------------- oracle workers
def _oracle_init(root):
    if root not in sys.path:
        sys.path.insert(0, root)
    lib()


def _worker_mixed_abs(payload, proposal, band):
    """(band, chi2, dchi2, dabs, dterm, dres), each (n_src, 7) after chi2, of
    the mixed oracle for one band, in a worker process."""
    L = lib()
    if not hasattr(L, "_mixed_abs_bound"):
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.fpo_evaluate_band_mixed_abs.argtypes = [ip, vp, vp, ip, vp, vp, vp, vp, vp]
        L.fpo_evaluate_band_mixed_abs.restype = ip
        L._mixed_abs_bound = True
    arrays, ns, nr = _resolve(payload)
    st = _struct_from_arrays(arrays, ns, nr)
    prop = np.ascontiguousarray(proposal)
    c = ctypes.c_double(0.0)
    g = np.zeros(ns * 7)
    a = np.zeros(ns * 7)
    t = np.zeros(ns * 7)
    rs = np.zeros(ns * 7)
    if L.fpo_evaluate_band_mixed_abs(band, st.ctypes.data, prop.ctypes.data, 1, ctypes.byref(c),
                                     g.ctypes.data, a.ctypes.data, t.ctypes.data,
                                     rs.ctypes.data) != 0:
        raise MemoryError("oracle allocation failed")
    return (band, c.value, g.reshape(ns, 7), a.reshape(ns, 7), t.reshape(ns, 7),
            rs.reshape(ns, 7))


def oracle_pool(processes):
    """A spawn pool of workers with the C oracle loaded."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    return ctx.Pool(processes, initializer=_oracle_init, initargs=(os.path.dirname(HERE),))


def mixed_abs_many(patch, jobs, pool, payload=None):
    """Mixed-oracle (band, chi2, dchi2, dabs, dterm, dres) for a list of
    (proposal, band) jobs, spread over `pool` (see oracle_pool)."""
    payload = payload or _patch_payload(patch)
    return pool.starmap(_worker_mixed_abs, [(payload, np.ascontiguousarray(p), b)
                                            for p, b in jobs])


def _worker_f64(payload, proposal, band, amps=None):
    """(band, chi2, dchi2 (n_src, 7)) of the all-FP64 oracle for one band, in a
    worker process; `amps` (n_sources, 10) float64 replaces the proposal's
    float amplitudes."""
    L = lib()
    arrays, ns, nr = _resolve(payload)
    st = _struct_from_arrays(arrays, ns, nr)
    prop = np.ascontiguousarray(proposal)
    c = ctypes.c_double(0.0)
    g = np.zeros(ns * 7)
    if amps is None:
        rc = L.fpo_evaluate_band_f64(band, st.ctypes.data, prop.ctypes.data, 1,
                                     ctypes.byref(c), g.ctypes.data, None)
    else:
        a = np.ascontiguousarray(amps, dtype=np.float64)
        fn = L.fpo_evaluate_band_f64_amps
        fn.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 3 + [ctypes.c_int] + \
            [ctypes.c_void_p] * 2
        fn.restype = ctypes.c_int
        rc = fn(band, st.ctypes.data, prop.ctypes.data, a.ctypes.data, 1, ctypes.byref(c),
                g.ctypes.data)
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return band, c.value, g.reshape(ns, 7)


def f64_chi2_many(patch, jobs, pool, payload=None):
    """All-FP64 chi2 for a list of (proposal, band[, amps]) jobs, spread over
    `pool` (`payload`: a patch_payload_file path, else the arrays are sent)."""
    return [c for c, _ in f64_many(patch, jobs, pool, payload)]


def f64_many(patch, jobs, pool, payload=None):
    """All-FP64 (chi2, dchi2) for a list of (proposal, band[, amps]) jobs."""
    payload = payload or _patch_payload(patch)
    args = [(payload, np.ascontiguousarray(j[0]), j[1], j[2] if len(j) > 2 else None)
            for j in jobs]
    return [(c, g) for _, c, g in pool.starmap(_worker_f64, args)]
