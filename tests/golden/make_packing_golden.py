"""Golden vectors for patch packing, made by the reference's own packing code.

Runs forcepho's ``StorePatch`` (forcepho/patches/pixel_patch.py:216-342:
find_exposures, find_pixels, pack_pix, _cap_snr) and ``Patch.pack_meta``
(forcepho/patches/patch.py:242-396: astrometry, flux calibration, PSF rows)
from the reference sources on a seeded synthetic store
(:func:`forcepho_b200.synth.make_store`), and writes their outputs to
``packing_store.npz`` next to this script.  Also packs the reference's test
image (tests/data/test_image in the reference) with its ``FITSPatch`` and
writes ``packing_fits.npz``.

The reference imports astropy and h5py, which this environment lacks.  This
script installs stand-ins for exactly the calls the packing path makes, all
of them this package's own readers: ``h5py.File`` -> forcepho_b200.h5lite,
``astropy.io.fits.getdata/getheader/Header.fromstring`` ->
forcepho_b200.fitsio, ``astropy.wcs.WCS`` -> forcepho_b200.wcs.TanWCS.  The
selection, ordering, concatenation, background, S/N cap and metadata
arithmetic are the reference's code.

Usage: python tests/golden/make_packing_golden.py [path/to/reference]
"""

import importlib
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from forcepho_b200 import fitsio, h5lite, synth  # noqa: E402
from forcepho_b200.wcs import TanWCS  # noqa: E402

# the cases of packing_store.npz: (name, region kind, region args, tweak_background, max_snr)
STORE_SEED = 11
STORE_CASES = [
    ("circle", "circle", (53.16, synth.DEC0, 2.5 / 3600.0), False, None),
    ("circle_bkg_snr", "circle", (53.1602, synth.DEC0 + 0.0003, 3.0 / 3600.0), "BKG", 100.0),
    ("rect", "rect", (53.1590, 53.1612, synth.DEC0 - 0.0006, synth.DEC0 + 0.0005), False, None),
]
STORE_KW = dict(n_bands=3, exposures_per_band=2, nside=256, super_pixel_size=8, n_sources=4)


def install_shims(ref):
    class FHeader(fitsio.Header):
        def fromstring(self, s, *a, **k):
            return fitsio.Header.fromstring(s)

    mods = {}

    def mod(name, **attrs):
        m = types.ModuleType(name)
        m.__path__ = []
        m.__dict__.update(attrs)
        mods[name] = m
        return m

    mod("astropy")
    mod("astropy.io", fits=mod("astropy.io.fits", Header=FHeader, getdata=fitsio.getdata,
                               getheader=fitsio.getheader))
    mod("astropy.wcs", WCS=TanWCS)
    mod("astropy.utils")
    mod("astropy.utils.exceptions", AstropyWarning=Warning)
    mod("h5py", File=lambda path, mode="r", **kw: h5lite.File(path))
    sys.modules.update(mods)
    pkg = types.ModuleType("forcepho")
    pkg.__path__ = [os.path.join(ref, "forcepho")]
    pkg.source_dir = os.path.join(ref, "forcepho", "src")
    sys.modules["forcepho"] = pkg
    for sub in ("patches", "utils"):   # skip package __init__s that pull in GPU/plot code
        m = types.ModuleType(f"forcepho.{sub}")
        m.__path__ = [os.path.join(ref, "forcepho", sub)]
        sys.modules[f"forcepho.{sub}"] = m
    sys.modules["forcepho.utils"].scale_at_sky = \
        importlib.import_module("forcepho.utils.wcs").scale_at_sky
    return importlib.import_module("forcepho.patches.pixel_patch"), \
        importlib.import_module("forcepho.region")


def region_of(region_mod, kind, args):
    return (region_mod.CircularRegion(*args) if kind == "circle"
            else region_mod.RectangularRegion(*args))


PIXEL_ARRAYS = ("data", "ierr", "xpix", "ypix")


def digest(a):
    """sha256 of a float32 array's bytes (the pixel arrays are compared bit
    for bit; a digest keeps the fixture small)."""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def packed(p, full_pixels=True):
    out = {k: np.asarray(getattr(p, k)) for k in
           ("exposure_start", "exposure_N", "band_start", "band_N", "D", "CW", "crpix", "crval",
            "G", "rad2", "n_psf_per_source", "psfgauss_start")}
    for k in PIXEL_ARRAYS:
        a = np.asarray(getattr(p, k), dtype=np.float32)
        if full_pixels:
            out[k] = a
        else:
            out[k + "_sha256"] = np.array(digest(a))
            out[k + "_head"] = a[:64]
    ps = np.asarray(p.psfgauss)
    out["psfgauss"] = np.stack([ps[c].astype(np.float64) for c in ps.dtype.names], -1)
    out["epaths"] = np.array([str(e) for e in p.epaths])
    out["reference_coordinates"] = np.asarray(p.patch_reference_coordinates)
    return out


def main(ref):
    pp, region_mod = install_shims(ref)
    spline = os.path.join(ref, "tests", "data", "sersic_splinedata_large.h5")
    res = {}
    with tempfile.TemporaryDirectory() as d:
        st = synth.make_store(d, seed=STORE_SEED, **STORE_KW)
        for name, kind, args, tweak, max_snr in STORE_CASES:
            p = pp.StorePatch(pixelstore=st["pixelstore"], metastore=st["metastore"],
                              psfstore=st["psfstore"], splinedata=spline)
            p.metastore.populate_wcs()
            p.max_snr = max_snr
            p.build_patch(region_of(region_mod, kind, args), st["catalog"],
                          allbands=st["bands"], tweak_background=tweak)
            for k, v in packed(p, full_pixels=False).items():
                res[f"{name}/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "packing_store.npz"), **res)
    print("packing_store.npz", len(res), "arrays")

    img = os.path.join(ref, "tests", "data", "test_image",
                       "sersic1.0_rhalf0.150_snr050_noise1_data.fits")
    psf = img.replace("_data.fits", "_psf.h5")
    cat = fitsio.getdata(img, -1)
    p = pp.FITSPatch(fitsfiles=[img], psfstore=psf, splinedata=spline, sci_ext=0, unc_ext=1,
                     return_residual=True)
    region = region_mod.CircularRegion(cat["ra"][0], cat["dec"][0],
                                       (cat["rhalf"][0] * 5 + 0.3) / 3600.0)
    p.build_patch(region, None, allbands=["CLEAR"])
    p.pack_meta(p.set_scene(cat))
    out = packed(p)
    out["catalog"] = np.array([[cat[c][0] for c in ("ra", "dec", "q", "pa", "sersic", "rhalf",
                                                    "CLEAR")]])
    out["region"] = np.array([region.ra, region.dec, region.radius])
    np.savez_compressed(os.path.join(HERE, "packing_fits.npz"), **out)
    print("packing_fits.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FPHO_REFERENCE")
    if not ref:
        sys.exit("usage: make_packing_golden.py <reference checkout> (or set FPHO_REFERENCE)")
    main(ref)
