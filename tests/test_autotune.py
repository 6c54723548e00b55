"""CPU: the autotuner's configuration cache (no GPU: the timing search is
replaced by a stand-in tuner).  A winner is stored under the workload's
signature and read back; a corrupt cache file, an entry that is not a dict,
and an entry naming a variant the library does not compile are all ignored
and re-tuned; a tuner that fails or returns an invalid configuration gives
the default."""
import json

import numpy as np
import pytest

from forcepho_b200 import _lib, autotune


class _P:
    def __init__(self, n_sources=3, npix=(4096, 4096), npsf=(5,)):
        self.n_sources = n_sources
        self.exposure_N = np.array(npix)
        self.n_psf_per_source = np.array(npsf)


@pytest.fixture
def cache(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setattr(autotune, "CACHE", str(path))
    return path


def _tuner(cfg, calls):
    def f():
        calls.append(1)
        return dict(cfg)
    return f


def test_single_round_trip_and_invalid_entries(cache):
    P = _P()
    good = {"variant": 3, "live_cap": 192, "schedule": 1}
    calls = []
    assert autotune.choose_config(P, tune_fn=_tuner(good, calls)) == good and len(calls) == 1
    assert json.loads(cache.read_text())[autotune.signature(P)] == good
    assert autotune.choose_config(P, tune_fn=_tuner(good, calls)) == good and len(calls) == 1
    # a variant the library does not compile: ignored, re-tuned
    cache.write_text(json.dumps({autotune.signature(P): {"variant": len(_lib.variants()) + 5,
                                                         "live_cap": 160, "schedule": 1}}))
    assert autotune.choose_config(P, tune_fn=_tuner(good, calls)) == good and len(calls) == 2
    # a corrupt file and a non-dict file
    for text in ("{not json", "[1, 2, 3]"):
        cache.write_text(text)
        assert autotune.choose_config(P, tune_fn=_tuner(good, calls)) == good
    assert len(calls) == 4
    # explicit arguments win without tuning
    assert autotune.choose_config(P, variant=0, live_cap=96, schedule=0,
                                  tune_fn=_tuner(good, calls)) == \
        {"variant": 0, "live_cap": 96, "schedule": 0} and len(calls) == 4


def test_single_failing_or_invalid_tuner_gives_default(cache):
    P = _P(n_sources=7)

    def boom():
        raise RuntimeError("no GPU")
    assert autotune.choose_config(P, tune_fn=boom) == autotune.DEFAULT
    bad = {"variant": -1, "live_cap": 160, "schedule": 1}
    assert autotune.choose_config(P, tune_fn=lambda: bad) == autotune.DEFAULT
    assert not cache.exists() or autotune.signature(P) not in json.loads(cache.read_text())


def test_batch_round_trip_and_signature(cache):
    from forcepho_b200.batch import batch_variants
    variants = batch_variants()
    assert 6 in variants and len(variants) >= 3
    patches = [_P(3), _P(20, npix=(128 * 128,) * 4)]
    good = {"variant": variants[-1], "live_cap": 128, "ctas_per_sm": 4}
    calls = []
    assert autotune.choose_batch_config(patches, tune_fn=_tuner(good, calls)) == good
    assert autotune.choose_batch_config(patches, tune_fn=_tuner(good, calls)) == good
    assert len(calls) == 1
    # a patch-only variant (no batched kernel) in the cache is re-tuned
    non_batch = [v for v in range(len(_lib.variants())) if v not in variants][0]
    cache.write_text(json.dumps({autotune.batch_signature(patches):
                                 {"variant": non_batch, "live_cap": 128, "ctas_per_sm": 0}}))
    assert autotune.choose_batch_config(patches, tune_fn=_tuner(good, calls)) == good
    assert len(calls) == 2
    assert autotune.batch_signature(patches) != autotune.batch_signature(patches[:1])
    assert autotune.choose_batch_config(patches[:1], tune_fn=lambda: {"variant": 6}) == \
        autotune.BATCH_DEFAULT


def test_candidates_cover_compiled_shapes():
    shapes = _lib.variant_shapes()
    assert len(shapes) == len(_lib.variants())
    cands = autotune.all_candidates()
    assert {c[0] for c in cands} == set(range(len(shapes)))
    assert any(sp > 0 for _, _, sp in shapes)        # Gaussian-split shapes are compiled
    bc = autotune.batch_candidates()
    assert {c[2] for c in bc} == set(autotune.BATCH_CTAS)
