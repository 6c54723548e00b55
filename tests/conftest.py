import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


GOLDEN_CASES = ["single_seed1", "single_seed7", "mini_3src_2band"]


def load_golden(name):
    """(patch, proposal, fixture dict) for a committed golden case."""
    from forcepho_b200.synth import SyntheticPatch
    from forcepho_b200.sources import default_table
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    P = SyntheticPatch()
    for k in ["data", "ierr", "xpix", "ypix", "exposure_start", "exposure_N", "band_start",
              "band_N", "rad2", "D", "crpix", "crval", "CW", "G", "n_psf_per_source", "psfgauss",
              "psfgauss_start"]:
        setattr(P, k, d[k])
    P.n_sources = int(d["n_sources"])
    P.n_radii = int(d["n_radii"])
    P.table = default_table()
    P.coerce_arrays()
    return P, d["proposal"], d
