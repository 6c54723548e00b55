"""Launch-configuration autotuner for the pixel-tile kernels.

The tile kernel is compiled in several variants (see ``fpho_variant_shape``:
threads per CTA, pixels per tile, and whether a tile's Gaussians are split
across warps), takes a shared-memory stage size (``live_cap``: image-Gaussian
records per staged chunk) and runs either one CTA per tile or as persistent
CTAs taking the costliest tiles first (``schedule``).  The batched kernel
(:class:`forcepho_b200.batch.PatchBatch`) is compiled for a subset of the
variants (``fpho_batch_variants``) and its persistent grid can be capped in
resident CTAs per SM (``ctas_per_sm``, 0 = as many as fit).  These are the
counterparts of the reference's fixed launch shape (``thread_block``,
``shared_size``, ``max_registers``; forcepho/proposal.py:62-65, 88-89).

The best choice depends on the patch (sources, PSF components, pixels per
exposure, source density) or on the batch.  :func:`choose_config` and
:func:`choose_batch_config` time the candidates on the workload itself with
CUDA events and cache the winner in a JSON file keyed by a coarse signature,
under a file lock for concurrent processes.  A cache entry that is not a
valid configuration of the library as compiled (a corrupt file, a variant
that no longer exists) is ignored and re-tuned.
"""

import fcntl
import json
import os

import numpy as np

from . import _lib

CACHE = os.environ.get("FPHO_AUTOTUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "forcepho_b200",
                                    "autotune.json"))
DEFAULT = {"variant": 8, "live_cap": 256, "schedule": 1}  # 4 warps share 256-pixel tiles
BATCH_DEFAULT = {"variant": 6, "live_cap": 128, "ctas_per_sm": 0}   # 64 threads x 8 pixels
LIVE_CAPS = (96, 128, 160, 192, 256, 384)
SCHEDULES = (0, 1)
BATCH_LIVE_CAPS = (96, 128, 192)
BATCH_CTAS = (0, 6)


# ------------------------------------------------------------------ signatures
def _pow2(n):
    return 1 << max(int(n) - 1, 0).bit_length()


def signature(patch):
    """Cache key of a single patch: sources, PSF components, pixels per exposure."""
    npix = int(np.median(patch.exposure_N)) if len(patch.exposure_N) else 0
    npsf = int(np.max(patch.n_psf_per_source)) if len(patch.n_psf_per_source) else 0
    return f"s{patch.n_sources}_g{npsf}_p{_pow2(npix)}"


def batch_signature(patches):
    """Cache key of a batch: patch count, and (rounded up to powers of two)
    the total pixels and sources and the largest PSF component count."""
    npix = sum(int(np.sum(p.exposure_N)) for p in patches)
    nsrc = sum(int(p.n_sources) for p in patches)
    npsf = max(int(np.max(p.n_psf_per_source)) for p in patches)
    return f"batch_n{len(patches)}_s{_pow2(nsrc)}_g{npsf}_p{_pow2(npix)}"


# ------------------------------------------------------------------ cache
def _load():
    try:
        with open(CACHE) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(key, value):
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    with open(CACHE + ".lock", "w") as lk:
        fcntl.flock(lk, fcntl.LOCK_EX)
        d = _load()
        d[key] = value
        tmp = CACHE + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE)


def _is_int(x):
    return isinstance(x, int) and not isinstance(x, bool)


def valid_config(c):
    """A single-patch configuration the compiled library can run."""
    return (isinstance(c, dict) and all(_is_int(c.get(k)) for k in ("variant", "live_cap",
                                                                    "schedule"))
            and 0 <= c["variant"] < len(_lib.variants()) and 32 <= c["live_cap"] <= 4096
            and c["schedule"] in SCHEDULES)


def valid_batch_config(c):
    """A batch configuration the compiled library can run."""
    from .batch import batch_variants
    return (isinstance(c, dict) and all(_is_int(c.get(k)) for k in ("variant", "live_cap",
                                                                    "ctas_per_sm"))
            and c["variant"] in batch_variants() and 32 <= c["live_cap"] <= 4096
            and 0 <= c["ctas_per_sm"] <= 32)


def _cached_or_tuned(key, valid, tune_fn, default, retune):
    if not retune:
        c = _load().get(key)
        if valid(c):
            return c
    try:
        best = tune_fn()
    except Exception:
        return dict(default)
    if not valid(best):
        return dict(default)
    try:
        _store(key, best)
    except OSError:
        pass
    return best


# ------------------------------------------------------------------ single patch
def time_config(patch, proposal_dev, outs, variant, live_cap, schedule=0, reps=5):
    """Median milliseconds of one evaluation with the given configuration."""
    import torch
    dp = patch.device_patch
    dp.set_config(variant, live_cap)
    dp.set_schedule(schedule)
    chi2, dchi2 = outs
    s = torch.cuda.current_stream()
    ns = patch.n_sources

    def ev():
        _lib.call("fpho_evaluate_proposal", dp.handle, proposal_dev.data_ptr(), ns,
                  chi2.data_ptr(), dchi2.data_ptr(), 7 * ns, 0, s.cuda_stream)

    ev()
    ev()  # the persistent schedule orders tiles by the previous evaluation's costs
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ev()
        e1.record(s)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def all_candidates():
    """Every (variant, live_cap, schedule) of the compiled library."""
    return [(v, lc, sc) for v in range(len(_lib.variants())) for lc in LIVE_CAPS
            for sc in SCHEDULES]


def tune(patch, proposal=None, candidates=None):
    """Time every (variant, live_cap, schedule) on `patch` (already on the
    device); returns (best config, {config: ms}).  Configurations the patch
    cannot run (shared memory) are skipped."""
    import torch
    proposal = patch.proposal() if proposal is None else proposal
    dprop = torch.from_numpy(np.ascontiguousarray(proposal).view(np.uint8).copy()).cuda()
    nb, ns = patch.n_bands, patch.n_sources
    outs = (torch.zeros(nb, dtype=torch.float64, device="cuda"),
            torch.zeros(nb * ns * 7, dtype=torch.float32, device="cuda"))
    cands = all_candidates() if candidates is None else candidates
    res = {}
    for cand in cands:
        v, lc = cand[0], cand[1]
        sc = cand[2] if len(cand) > 2 else 0
        try:
            res[(v, lc, sc)] = time_config(patch, dprop, outs, v, lc, sc)
        except _lib.FphoError:
            continue
    best = min(res, key=res.get)
    return {"variant": best[0], "live_cap": best[1], "schedule": best[2]}, res


def choose_config(patch, variant=None, live_cap=None, schedule=None, retune=False,
                  tune_fn=None):
    """Configuration for `patch`: explicit arguments win, else the cached
    winner for its signature, else tune now (the patch must be on the
    device).  `tune_fn() -> config` replaces the timing search."""
    if variant is not None:
        return {"variant": int(variant), "live_cap": int(live_cap or DEFAULT["live_cap"]),
                "schedule": int(DEFAULT["schedule"] if schedule is None else schedule)}
    tune_fn = tune_fn or (lambda: tune(patch)[0])
    return _cached_or_tuned(signature(patch), valid_config, tune_fn, DEFAULT, retune)


def apply_config(patch, cfg):
    """Set a configuration from :func:`choose_config` on the patch's handle."""
    patch.device_patch.set_config(cfg["variant"], cfg["live_cap"])
    patch.device_patch.set_schedule(cfg.get("schedule", 0))


# ------------------------------------------------------------------ batches
def batch_candidates():
    """Every (variant, live_cap, ctas_per_sm) the batched kernel is compiled for."""
    from .batch import batch_variants
    return [(v, lc, c) for v in batch_variants() for lc in BATCH_LIVE_CAPS for c in BATCH_CTAS]


def time_batch(patches, variant, live_cap, ctas_per_sm, reps=5):
    """Median milliseconds of one batched evaluation of `patches` (on the
    device) with the given configuration."""
    import torch
    from .batch import PatchBatch
    b = PatchBatch(patches, live_cap=live_cap, variant=variant, ctas_per_sm=ctas_per_sm)
    try:
        dprop, chi2, dchi2 = b.device_buffers()
        s = torch.cuda.current_stream()
        for _ in range(2):
            b.evaluate_device(dprop, chi2, dchi2)
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            b.evaluate_device(dprop, chi2, dchi2)
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))
    finally:
        b.free()


def tune_batch(patches, candidates=None, reps=5):
    """Time every (variant, live_cap, ctas_per_sm) on the batch; returns
    (best config, {config: ms}).  The patches end up planned for the last
    candidate timed: build the batch from the result afterwards."""
    cands = batch_candidates() if candidates is None else candidates
    res = {}
    for v, lc, c in cands:
        try:
            res[(v, lc, c)] = time_batch(patches, v, lc, c, reps=reps)
        except _lib.FphoError:
            continue
    best = min(res, key=res.get)
    return {"variant": best[0], "live_cap": best[1], "ctas_per_sm": best[2]}, res


def choose_batch_config(patches, retune=False, tune_fn=None):
    """Configuration for a batch of `patches` (on the device): the cached
    winner for its signature, else tune now.  `tune_fn() -> config`
    replaces the timing search."""
    tune_fn = tune_fn or (lambda: tune_batch(patches)[0])
    return _cached_or_tuned(batch_signature(patches), valid_batch_config, tune_fn,
                            BATCH_DEFAULT, retune)
