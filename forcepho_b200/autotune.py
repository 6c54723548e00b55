"""Launch-configuration autotuner for the pixel-tile kernel.

The tile kernel is compiled in several variants (threads per CTA x pixels per
thread, see ``fpho_variant_info``), takes a shared-memory stage size
(``live_cap``: image-Gaussian records per staged chunk) and runs either one
CTA per tile or as persistent CTAs taking the costliest tiles first
(``schedule``, ``fpho_patch_set_schedule``).  The best choice depends on the
patch (sources, PSF components, pixels per exposure, source density).
:func:`choose_config` times every candidate on the patch itself with CUDA
events and caches the winner in a JSON file keyed by a coarse signature of the
patch, guarded by a lock for concurrent processes.
"""

import fcntl
import json
import os

import numpy as np

from . import _lib

CACHE = os.environ.get("FPHO_AUTOTUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "forcepho_b200",
                                    "autotune.json"))
DEFAULT = {"variant": 3, "live_cap": 160, "schedule": 1}   # 64 threads x 4 pixels
LIVE_CAPS = (96, 128, 160, 192, 256, 384)
SCHEDULES = (0, 1)


def signature(patch):
    npix = int(np.median(patch.exposure_N)) if len(patch.exposure_N) else 0
    npsf = int(np.max(patch.n_psf_per_source)) if len(patch.n_psf_per_source) else 0
    return f"s{patch.n_sources}_g{npsf}_p{1 << max(npix - 1, 0).bit_length()}"


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
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


def tune(patch, proposal=None, candidates=None):
    """Time every (variant, live_cap, schedule) on `patch` (already on the
    device); returns (best config, {config: ms})."""
    import torch
    proposal = patch.proposal() if proposal is None else proposal
    dprop = torch.from_numpy(np.ascontiguousarray(proposal).view(np.uint8).copy()).cuda()
    nb, ns = patch.n_bands, patch.n_sources
    outs = (torch.zeros(nb, dtype=torch.float64, device="cuda"),
            torch.zeros(nb * ns * 7, dtype=torch.float32, device="cuda"))
    if candidates is None:
        candidates = []
        for v, (nt, k) in enumerate(_lib.variants()):
            for lc in LIVE_CAPS:
                for sc in SCHEDULES:
                    candidates.append((v, lc, sc))
    res = {}
    for cand in candidates:
        v, lc = cand[0], cand[1]
        sc = cand[2] if len(cand) > 2 else 0
        try:
            res[(v, lc, sc)] = time_config(patch, dprop, outs, v, lc, sc)
        except _lib.FphoError:
            continue
    best = min(res, key=res.get)
    return {"variant": best[0], "live_cap": best[1], "schedule": best[2]}, res


def choose_config(patch, variant=None, live_cap=None, schedule=None, retune=False):
    """Configuration for `patch`: explicit arguments win, else the cached
    winner for its signature, else tune now (patch must be on the device)."""
    if variant is not None:
        return {"variant": int(variant), "live_cap": int(live_cap or DEFAULT["live_cap"]),
                "schedule": int(DEFAULT["schedule"] if schedule is None else schedule)}
    key = signature(patch)
    if not retune:
        c = _load().get(key)
        if c and c.get("variant", 99) < len(_lib.variants()) and "schedule" in c:
            return c
    try:
        best, _ = tune(patch)
    except Exception:
        return dict(DEFAULT)
    try:
        _store(key, best)
    except OSError:
        pass
    return best


def apply_config(patch, cfg):
    """Set a configuration from :func:`choose_config` on the patch's handle."""
    patch.device_patch.set_config(cfg["variant"], cfg["live_cap"])
    patch.device_patch.set_schedule(cfg.get("schedule", 0))
