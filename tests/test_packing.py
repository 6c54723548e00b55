"""CPU: the packing path's host pieces against the reference's own packing code.

tests/golden/packing_store.npz and packing_fits.npz were written by
tests/golden/make_packing_golden.py, which runs forcepho's StorePatch,
FITSPatch and Patch.pack_meta from the reference sources.  Checked here:

  * the HDF5 subset reader (on the reference's own data files when present)
    and writer (round trips: nested groups, B-trees of several levels,
    compound and array types, attributes);
  * the FITS reader, the TAN WCS and the region helpers;
  * the host StorePatch / FITSPatch mirrors, bit for bit against the golden
    pixel digests, index arrays and metadata;
  * oracle/packing.py (the checker of the device store) against the same
    digests.
"""
import hashlib
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
# the reference checkout's test data, when FPHO_REFERENCE names a checkout
REF_DATA = os.path.join(os.environ.get("FPHO_REFERENCE", "/nonexistent"), "tests", "data")


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def _cases():
    import sys
    sys.path.insert(0, GOLDEN)
    import make_packing_golden as G
    return G


@pytest.fixture(scope="module")
def store(tmp_path_factory):
    from forcepho_b200 import synth
    G = _cases()
    return synth.make_store(str(tmp_path_factory.mktemp("store")), seed=G.STORE_SEED,
                            **G.STORE_KW)


def _region(kind, args):
    from forcepho_b200.region import CircularRegion, RectangularRegion
    return CircularRegion(*args) if kind == "circle" else RectangularRegion(*args)


# ------------------------------------------------------------------ HDF5
def test_h5_roundtrip(tmp_path):
    from forcepho_b200 import h5lite
    from forcepho_b200.patches.patch import PSF_DTYPE
    rng = np.random.default_rng(0)
    arr = np.dtype([("gauss_params", np.float32, 6), ("sersic_bin", np.int32)])
    P = np.zeros((3, 9), dtype=arr)
    P["gauss_params"] = rng.normal(size=(3, 9, 6))
    P["sersic_bin"] = np.arange(9)
    Q = np.zeros((2, 4), dtype=PSF_DTYPE)
    Q["amp"] = rng.random((2, 4))
    ds = {f"F090W/exp{e:03d}/data": rng.normal(size=(2, 2, 8)).astype(np.float32)
          for e in range(300)}
    ds.update({"CLEAR/parameters": P, "CLEAR/q": Q, "x": np.arange(5, dtype=np.int16),
               "s": np.float64(3.5), "u": np.arange(4, dtype=np.uint64).reshape(2, 2)})
    attrs = {"/": {"nside_full": np.array([32, 32]), "super_pixel_size": 8, "name": "store"},
             "CLEAR": {"n_psf_per_source": np.int64(9)},
             "F090W/exp003/data": {"counts_to_flux": 1.5, "flux_units": "nJy"}}
    path = str(tmp_path / "t.h5")
    h5lite.write(path, ds, attrs)
    data, at = h5lite.read_tree(path)
    for k, v in ds.items():
        got = np.asarray(data[k])
        assert got.dtype == np.asarray(v).dtype and np.array_equal(got, v), k
    assert at["/"]["super_pixel_size"] == 8 and at["/"]["name"] == "store"
    assert list(at["/"]["nside_full"]) == [32, 32]
    assert at["CLEAR"]["n_psf_per_source"] == 9
    assert at["F090W/exp003/data"] == {"counts_to_flux": 1.5, "flux_units": "nJy"}
    with h5lite.File(path) as f:
        assert len(f["F090W"].keys()) == 300
        assert f["F090W"].keys() == sorted(f["F090W"].keys())
        assert "F090W/exp299/data" in f and "F090W/exp300/data" not in f
        assert isinstance(f["F090W/exp007/data"].array(), np.memmap)


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data files not present")
def test_h5_reads_reference_files():
    from forcepho_b200 import h5lite
    from forcepho_b200.patches.storage import PSFStore
    with h5lite.File(f"{REF_DATA}/sersic_splinedata_large.h5") as f:
        assert sorted(f.keys()) == ["amplitudes", "nsersic", "radii", "rh"]
        assert f["amplitudes"].shape == (5555, 9) and f["radii"].shape == (9,)
    with h5lite.File(f"{REF_DATA}/sersic_mog_model.smooth=0.0150.h5") as f:
        assert f.attrs["smoothing"] == 0.015
        assert f["model"].shape == (50, 6399)
    psf = PSFStore(f"{REF_DATA}/test_image/sersic1.0_rhalf0.150_snr050_noise1_psf.h5")
    rows = psf.lookup("CLEAR")
    assert psf.n_psf_per_source("CLEAR") == 9 and len(rows) == 9
    assert np.array_equal(rows["sersic_bin"], np.arange(9))
    assert np.all(rows["Cxx"] == 6.25) and np.all(rows["amp"] == 1.0)


# ------------------------------------------------------------------ FITS, WCS, regions
def test_fits_header_roundtrip_and_wcs():
    from forcepho_b200 import synth
    from forcepho_b200.fitsio import Header
    from forcepho_b200.wcs import TanWCS, scale_at_sky
    h = Header(synth.store_header("F200W", (2048, 2048), (53.1, -27.8), (1024.3, 1020.7), 17.0))
    h2 = Header.fromstring(h.tostring())
    assert h2 == h
    w = TanWCS(h2)
    x0, y0 = w.world_to_pixel_values(53.1, -27.8)
    assert abs(x0 - 1023.3) < 1e-9 and abs(y0 - 1019.7) < 1e-9
    xy = np.random.default_rng(1).uniform(-3000, 5000, (2, 500))
    back = np.array(w.world_to_pixel_values(*w.pixel_to_world_values(*xy)))
    assert np.abs(back - xy).max() < 1e-7
    CW, D = scale_at_sky((53.1005, -27.8002), w)
    assert np.allclose(np.linalg.inv(D) / 3600.0, w.cd, rtol=1e-12)
    # the finite-difference branch also sees the projection's local rotation
    # (meridian convergence, ~1e-5 of the scale 60 px from the tangent point)
    w.has_distortion = True
    CW2, D2 = scale_at_sky((53.1005, -27.8002), w)
    assert np.abs(CW2 - CW).max() < 1e-5 * np.abs(CW).max()
    assert np.abs(D2 - D).max() < 1e-5 * np.abs(D).max()


def test_regions():
    from forcepho_b200.region import RectangularRegion, polygon_contains, polygons_overlap
    a = RectangularRegion(58, 59, 26, 27)
    assert polygons_overlap(a, RectangularRegion(57, 60, 25, 28))
    assert not polygons_overlap(a, RectangularRegion(60, 62, 25, 28))
    assert polygons_overlap(a, RectangularRegion(58.5, 62, 25, 28))
    pts = np.atleast_2d([[0.5, 0.5], [0.5, 1.1], [-0.1, 0.5]])
    for poly, want in (([[0, 0], [1., 0], [1, 1], [0, 1]], [True, False, False]),
                       ([[0, 0], [0., 1], [1, 1], [1, 0]], [True, False, False]),
                       ([[0, 0], [0, 3.0], [1, 1], [1, 0]], [True, True, False])):
        assert list(polygon_contains(np.array(poly), pts)) == want


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data files not present")
def test_fits_reader_on_reference_image():
    from forcepho_b200 import fitsio
    hdus = fitsio.read_hdus(f"{REF_DATA}/test_image/sersic1.0_rhalf0.150_snr050_noise1_data.fits")
    assert [d.shape for _, d in hdus[:3]] == [(100, 100)] * 3
    cat = hdus[-1][1]
    assert cat["ra"][0] == 53.0 and cat["dec"][0] == -27.0 and cat["rhalf"][0] == 0.15
    assert hdus[0][0]["CTYPE1"] == "RA---TAN" and hdus[0][0]["FILTER"] == "CLEAR"


# ------------------------------------------------------------------ packing vs the reference
def _check_packed(p, gold, name):
    for k in ("data", "ierr", "xpix", "ypix"):
        assert _digest(getattr(p, k)) == str(gold[f"{name}/{k}_sha256"]), (name, k)
    for k in ("exposure_start", "exposure_N", "band_start", "band_N", "D", "CW", "crpix",
              "crval", "G", "rad2", "n_psf_per_source", "psfgauss_start"):
        np.testing.assert_array_equal(np.asarray(getattr(p, k)), gold[f"{name}/{k}"],
                                      err_msg=f"{name}/{k}")
    ps = np.stack([p.psfgauss[c].astype(np.float64) for c in p.psfgauss.dtype.names], -1)
    np.testing.assert_array_equal(ps, gold[f"{name}/psfgauss"])
    assert list(p.epaths) == [str(e) for e in gold[f"{name}/epaths"]]


def test_store_patch_matches_reference(store):
    from forcepho_b200.patches.pixel_patch import StorePatch
    G = _cases()
    gold = np.load(os.path.join(GOLDEN, "packing_store.npz"))
    for name, kind, args, tweak, max_snr in G.STORE_CASES:
        p = StorePatch(store["pixelstore"], store["metastore"], store["psfstore"])
        p.max_snr = max_snr
        p.build_patch(_region(kind, args), store["catalog"], allbands=store["bands"],
                      tweak_background=tweak)
        _check_packed(p, gold, name)


def test_oracle_packing_matches_reference(store):
    from oracle import packing as OP
    from forcepho_b200.patches.storage import MetaStore, PixelStore
    G = _cases()
    gold = np.load(os.path.join(GOLDEN, "packing_store.npz"))
    ps, ms = PixelStore(store["pixelstore"]), MetaStore(store["metastore"])
    for name, kind, args, tweak, max_snr in G.STORE_CASES:
        region = _region(kind, args)
        epaths = [str(e) for e in gold[f"{name}/epaths"]]
        sps, regs, bg = [], [], []
        for ep in epaths:
            band, exp = ep.split("/")
            w = ms.get_wcs(band, exp)
            sps.append(np.asarray(ps.data[ep + "/data"].array()))
            regs.append(region.device_params(w))
            bg.append(ms.headers[band][exp]["BKG"])
        out = OP.pack(sps, regs, background=bg if tweak else None, max_snr=max_snr)
        for k in ("data", "ierr", "xpix", "ypix"):
            assert _digest(out[k]) == str(gold[f"{name}/{k}_sha256"]), (name, k)
        np.testing.assert_array_equal(out["exposure_N"], gold[f"{name}/exposure_N"])
        np.testing.assert_array_equal(out["exposure_start"], gold[f"{name}/exposure_start"])


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data files not present")
def test_fits_patch_matches_reference():
    from forcepho_b200 import fitsio
    from forcepho_b200.patches.pixel_patch import FITSPatch
    from forcepho_b200.region import CircularRegion
    gold = np.load(os.path.join(GOLDEN, "packing_fits.npz"))
    img = f"{REF_DATA}/test_image/sersic1.0_rhalf0.150_snr050_noise1_data.fits"
    p = FITSPatch(fitsfiles=[img], psfstore=img.replace("_data.fits", "_psf.h5"),
                  splinedata=f"{REF_DATA}/sersic_splinedata_large.h5", sci_ext=0, unc_ext=1)
    p.build_patch(CircularRegion(*gold["region"]), None, allbands=["CLEAR"])
    p.pack_meta(p.set_scene(fitsio.getdata(img, -1)))
    for k in ("data", "ierr", "xpix", "ypix", "exposure_start", "exposure_N", "band_start",
              "band_N", "D", "CW", "crpix", "crval", "G", "rad2", "n_psf_per_source"):
        np.testing.assert_array_equal(np.asarray(getattr(p, k)), gold[k], err_msg=k)


def test_superpixelize_matches_the_loop():
    """The reshape in PixelStore.superpixelize gives the element order of
    the reference's double loop (storage.py:245-276), restated here."""
    from forcepho_b200.patches.storage import PixelStore
    rng = np.random.default_rng(3)
    im, ie = rng.normal(size=(24, 40)), rng.normal(size=(24, 40))
    ps = PixelStore.__new__(PixelStore)
    ps.super_pixel_size, ps.pix_dtype = 8, np.float32
    got = ps.superpixelize(im, ie)
    want = np.empty((3, 5, 128), dtype=np.float32)
    for ii in range(3):
        for jj in range(5):
            want[ii, jj, :64] = im[ii * 8:ii * 8 + 8, jj * 8:jj * 8 + 8].flatten()
            want[ii, jj, 64:] = ie[ii * 8:ii * 8 + 8, jj * 8:jj * 8 + 8].flatten()
    np.testing.assert_array_equal(got, want)


def test_pixelstore_add_exposure(tmp_path):
    """PixelStore.add_exposure as forcepho/patches/storage.py:151-243:
    background subtracted, masked and non-finite pixels get ierr = 0 and the
    background value as flux, then super-pixel order; existing paths are
    replaced."""
    from forcepho_b200.patches.storage import ImageSet, PixelStore
    rng = np.random.default_rng(8)
    path = str(tmp_path / "pix.h5")
    ps = PixelStore(path, nside_full=32, super_pixel_size=8)
    im = rng.normal(size=(32, 32)).astype(np.float32)
    ierr = np.abs(rng.normal(size=(32, 32))).astype(np.float32) + 0.5
    bkg = np.full((32, 32), 0.25, dtype=np.float32)
    mask = np.zeros((32, 32), dtype=np.int32)
    mask[3, 4] = 4
    im[5, 6] = np.nan
    ierr[7, 8] = -1.0
    ps.add_exposure(ImageSet(im=im.copy(), ierr=ierr.copy(), mask=mask, bkg=bkg, hdr={},
                             band="F200W", expID="e1", names="e1.fits"), bitmask=4)
    ps2 = PixelStore(path)
    assert list(np.asarray(ps2.nside_full).reshape(-1)) in ([32], [32, 32])
    assert ps2.super_pixel_size == 8
    sp = ps2.data["F200W/e1/data"][:]
    want_im, want_ie = im - bkg, ierr.copy()
    bad = np.zeros_like(mask, dtype=bool)
    bad[3, 4] = bad[5, 6] = bad[7, 8] = True
    want_ie[bad] = 0.0
    want_im[bad] = bkg[bad]
    np.testing.assert_array_equal(sp, ps2.superpixelize(want_im, want_ie))
    assert ps2.data["F200W/e1/data"].attrs["image_name"] == "e1.fits"
    ps2.add_exposure(ImageSet(im=np.ones_like(im), ierr=np.ones_like(ierr), mask=None, bkg=None,
                              hdr={},
                              band="F200W", expID="e1", names=None))
    ps2.close()
    assert np.all(PixelStore(path).data["F200W/e1/data"][:] == 1.0)
    assert PixelStore(path).exposure_paths() == ["F200W/e1"]


def test_direct_patch_and_metastore(store):
    """DirectPatch packs given arrays in header order; MetaStore finds the
    exposures whose footprint holds a sky position; Region.overlaps."""
    from forcepho_b200.patches.pixel_patch import DirectPatch
    from forcepho_b200.patches.storage import MetaStore, PixelStore
    from forcepho_b200.region import CircularRegion, RectangularRegion
    ms, ps = MetaStore(store["metastore"]), PixelStore(store["pixelstore"])
    s2 = ps.super_pixel_size ** 2
    pix, hdrs = {}, {}
    for ep in store["epaths"][:3]:
        band, exp = ep.split("/")
        sp = ps.data[ep + "/data"][:][:4, :4]
        pix[ep] = dict(flux=sp[..., :s2].reshape(-1), ierr=sp[..., s2:].reshape(-1),
                       xpix=ps.xpix[:4, :4].reshape(-1), ypix=ps.ypix[:4, :4].reshape(-1))
        hdrs[ep] = ms.headers[band][exp]
    p = DirectPatch(pixel_dict=pix, header_dict=hdrs, psfstore=store["psfstore"])
    p.build_patch(None, store["catalog"], allbands=store["bands"])
    assert list(p.epaths) == store["epaths"][:3]
    np.testing.assert_array_equal(p.exposure_N, [16 * s2] * 3)
    np.testing.assert_array_equal(p.data, np.concatenate([pix[e]["flux"] for e in p.epaths]))
    np.testing.assert_array_equal(p.band_N, [2, 1])
    assert p.D.shape == (3, len(store["catalog"]), 2, 2)
    ids, bands = ms.find_exposures((53.16, -27.78), store["bands"])
    assert len(ids) == len(store["epaths"])          # every dithered exposure covers the centre
    ids, _ = ms.find_exposures((53.16 + 1.0, -27.78), store["bands"])
    assert ids == []
    hdr = ms.headers[store["bands"][0]]["exp00"]
    assert CircularRegion(53.16, -27.78, 1.0 / 3600).overlaps(hdr)
    assert not RectangularRegion(54.0, 54.1, -27.0, -26.9).overlaps(hdr)


def test_tan_sip_wcs():
    """TAN-SIP (Shupe et al. 2005): zero coefficients give TAN exactly; the
    sky-to-pixel Newton inversion round-trips a distortion of several pixels
    to 1e-8 px, from the inverse polynomials when present; scale_at_sky takes
    the finite-difference branch and matches the local Jacobian."""
    from forcepho_b200 import synth
    from forcepho_b200.wcs import TanWCS, scale_at_sky
    h = synth.store_header("F200W", (2048, 2048), (53.1, -27.8), (1024.3, 1020.7), 17.0)
    h0 = dict(h, CTYPE1="RA---TAN-SIP", CTYPE2="DEC--TAN-SIP", A_ORDER=3, B_ORDER=3)
    w, w0 = TanWCS(h), TanWCS(h0)
    xy = np.random.default_rng(1).uniform(-100, 2100, (2, 400))
    np.testing.assert_array_equal(np.array(w.pixel_to_world_values(*xy)),
                                  np.array(w0.pixel_to_world_values(*xy)))
    h1 = dict(h0, A_2_0=2e-6, A_1_1=-3e-6, A_0_2=1e-6, A_3_0=4e-10, B_2_0=-1e-6, B_0_2=3e-6,
              B_1_2=-2e-10)
    w1 = TanWCS(h1)
    assert w1.has_distortion and not w.has_distortion
    rd = w1.pixel_to_world_values(*xy)
    assert np.abs(np.array(w.world_to_pixel_values(*rd)) - xy).max() > 3.0
    np.testing.assert_allclose(np.array(w1.world_to_pixel_values(*rd)), xy, rtol=0, atol=1e-8)
    h2 = dict(h1, AP_ORDER=2, BP_ORDER=2, AP_2_0=-2e-6, AP_1_1=3e-6, AP_0_2=-1e-6, BP_2_0=1e-6,
              BP_0_2=-3e-6)
    np.testing.assert_allclose(np.array(TanWCS(h2).world_to_pixel_values(*rd)), xy, rtol=0,
                               atol=1e-8)
    sky = (53.1003, -27.7996)
    CW, D = scale_at_sky(sky, w1)
    x0, y0 = w1.world_to_pixel_values(*sky)
    d = 1e-3
    J = np.array([np.subtract(w1.pixel_to_world_values(x0 + d, y0),
                              w1.pixel_to_world_values(x0 - d, y0)),
                  np.subtract(w1.pixel_to_world_values(x0, y0 + d),
                              w1.pixel_to_world_values(x0, y0 - d))]).T / (2 * d)
    np.testing.assert_allclose(CW, np.linalg.inv(J), rtol=1e-4)
    with pytest.raises(NotImplementedError):
        TanWCS(dict(h, CTYPE1="RA---TPV", CTYPE2="DEC--TPV"))


def test_store_patch_with_sip_headers(tmp_path):
    """A store whose headers carry SIP distortion packs on the host: the
    super-pixels selected are those whose corners the SIP-aware WCS puts in
    the circle, and the astrometry uses the finite-difference scale."""
    from oracle import packing as OP
    from forcepho_b200 import synth
    from forcepho_b200.patches.pixel_patch import StorePatch
    from forcepho_b200.region import CircularRegion
    st = synth.make_store(str(tmp_path), seed=5, sip=True, n_bands=2, exposures_per_band=2)
    p = StorePatch(st["pixelstore"], st["metastore"], st["psfstore"])
    region = CircularRegion(53.16, -27.78, 2.5 / 3600)
    p.build_patch(region, st["catalog"], allbands=st["bands"])
    assert all(w.has_distortion for w in p.wcses)
    sps = [np.asarray(p.pixelstore.data[e + "/data"].array()) for e in p.epaths]
    want = OP.pack(sps, [region.device_params(w) for w in p.wcses])
    for k in ("data", "ierr", "xpix", "ypix"):
        np.testing.assert_array_equal(getattr(p, k), want[k], err_msg=k)
    assert np.all(np.isfinite(p.CW)) and np.all(np.isfinite(p.crpix))


def test_h5_random_trees_roundtrip(tmp_path):
    """Random trees of groups and datasets (dtypes, shapes incl. scalars and
    empty arrays, attributes) survive h5lite.write -> h5lite.read_tree."""
    from hypothesis import given, settings, strategies as stn
    from forcepho_b200 import h5lite

    dtypes = [np.int8, np.uint16, np.int32, np.int64, np.float32, np.float64]
    names = stn.text(alphabet="abcdefghijklmnopqrstuvwxyz0123456789_", min_size=1, max_size=8)

    @settings(max_examples=25, deadline=None, derandomize=True)
    @given(stn.dictionaries(stn.lists(names, min_size=1, max_size=3).map("/".join),
                            stn.tuples(stn.sampled_from(dtypes),
                                       stn.lists(stn.integers(0, 5), max_size=3),
                                       stn.integers(0, 2 ** 31)),
                            min_size=1, max_size=12),
           stn.floats(allow_nan=False, allow_infinity=False), stn.integers(-2 ** 40, 2 ** 40))
    def check(spec, fattr, iattr):
        # a path may not be both a dataset and a group
        paths = sorted(spec)
        keep = [p for p in paths if not any(q.startswith(p + "/") for q in paths)]
        ds = {}
        for p in keep:
            dt, shape, seed = spec[p]
            rng = np.random.default_rng(seed)
            a = (rng.normal(size=shape) * 100).astype(dt) if shape else dt(rng.integers(0, 100))
            ds[p] = a
        path = str(tmp_path / "r.h5")
        h5lite.write(path, ds, {"/": {"f": fattr, "i": iattr, "s": "x"}})
        data, attrs = h5lite.read_tree(path)
        assert set(data) == set(ds)
        for p, a in ds.items():
            got = np.asarray(data[p])
            assert got.dtype == np.asarray(a).dtype and got.shape == np.shape(a), p
            np.testing.assert_array_equal(got, a)
        assert attrs["/"]["f"] == fattr and attrs["/"]["i"] == iattr and attrs["/"]["s"] == "x"

    check()


def test_wcs_random_roundtrip():
    """Random TAN and TAN-SIP WCSs (rotation, scale, reference point, pole
    distance) map pixels to the sky and back to 1e-7 px."""
    from hypothesis import given, settings, strategies as stn
    from forcepho_b200 import synth
    from forcepho_b200.wcs import TanWCS

    @settings(max_examples=60, deadline=None, derandomize=True)
    @given(stn.floats(0.0, 359.9), stn.floats(-85.0, 85.0), stn.floats(-180.0, 180.0),
           stn.floats(0.01, 0.2), stn.booleans(), stn.integers(0, 2 ** 31))
    def check(ra0, dec0, rot, scale, sip, seed):
        rng = np.random.default_rng(seed)
        h = synth.store_header("F200W", (2048, 2048), (ra0, dec0), (1024.5, 1000.0), rot,
                               scale=scale)
        if sip:
            h.update(CTYPE1="RA---TAN-SIP", CTYPE2="DEC--TAN-SIP", A_ORDER=2, B_ORDER=2,
                     A_2_0=rng.normal(0, 1e-6), A_1_1=rng.normal(0, 1e-6),
                     B_0_2=rng.normal(0, 1e-6))
        w = TanWCS(h)
        xy = rng.uniform(-500, 2500, (2, 50))
        back = np.array(w.world_to_pixel_values(*w.pixel_to_world_values(*xy)))
        assert np.abs(back - xy).max() < 1e-7

    check()


def test_store_helpers(store, tmp_path):
    """MetaStore write/read round trip, header_to_id (storage.py:39-57) and
    PSFStore's nearest-detector-location lookup (storage.py:548-562)."""
    from forcepho_b200.patches.storage import MetaStore, PSFStore, header_to_id
    ms = MetaStore(store["metastore"])
    out = str(tmp_path / "meta2.json")
    ms.write_to_file(out)
    ms2 = MetaStore(out)
    assert ms2.headers == ms.headers and ms2.nexp == ms.nexp == len(store["epaths"])
    hdr = {"FILTER": "F444W", "DETECTOR": "NRCALONG"}
    assert header_to_id(hdr, "/data/frames/sub/jw001_cal.fits") == ("F444W", "jw001_cal")
    assert header_to_id(hdr, "/data/frames/sub/jw001_cal.fits",
                        framedir="/data/frames") == ("F444W", "sub/jw001_cal")
    assert header_to_id(hdr, "x.fits", split_by_detector=["F444W"]) == ("F444WA", "x")
    psf = PSFStore(store["psfstore"])
    band = store["bands"][0]
    locs = np.asarray(psf.data[band]["detector_locations"][:])
    pars = psf.data[band]["parameters"][:]
    for k in range(locs.shape[1]):
        rows = psf.lookup(band, xy=(locs[0, k] + 0.1, locs[1, k] - 0.1))
        np.testing.assert_array_equal(rows["amp"], pars[k]["amp"])
    np.testing.assert_array_equal(psf.lookup(band)["Cxx"], pars[0]["Cxx"])
    assert psf.n_psf_per_source(band) == pars.shape[1]


def test_h5_streamed_write_in_blocks(tmp_path, monkeypatch):
    """Dataset contents are streamed to the file in blocks (here forced to 1000
    bytes) and a rewrite reads the old datasets through memory maps."""
    from forcepho_b200 import h5lite
    from forcepho_b200.patches.storage import PixelStore
    monkeypatch.setattr(h5lite._Out.save, "__defaults__", (1000,))
    rng = np.random.default_rng(2)
    big = rng.normal(size=(37, 11, 29)).astype(np.float64)
    path = str(tmp_path / "s.h5")
    h5lite.write(path, {"g/big": big, "g/small": np.arange(3, dtype=np.int16)})
    data, _ = h5lite.read_tree(path, memmap=True)
    assert isinstance(data["g/big"], np.memmap)
    np.testing.assert_array_equal(data["g/big"], big)
    ps = PixelStore(str(tmp_path / "p.h5"), nside_full=16, super_pixel_size=8)
    sp = [rng.normal(size=(2, 2, 128)).astype(np.float32) for _ in range(3)]
    for i, a in enumerate(sp):
        ps.write_exposures({f"F200W/e{i}": (a, {"k": i})})
    ps2 = PixelStore(str(tmp_path / "p.h5"))
    for i, a in enumerate(sp):
        np.testing.assert_array_equal(ps2.data[f"F200W/e{i}/data"][:], a)
        assert ps2.data[f"F200W/e{i}/data"].attrs["k"] == i


def test_result_h5_roundtrip(tmp_path):
    """fitting.Result.dump_to_h5 / read_from_h5 as forcepho's Result
    (fitting.py:186-218): arrays as datasets, scalars and strings as
    attributes, anything else reported."""
    from forcepho_b200.fitting import Result
    r = Result(ndim=7, chain=np.arange(21.0).reshape(3, 7), wall_time=1.5, message="ok",
               accept=np.array([0.8, 0.7]), sampler=object())
    msgs = r.dump_to_h5(str(tmp_path / "out" / "r.h5"))
    assert len(msgs) == 1 and "sampler" in msgs[0]
    back = Result(filename=str(tmp_path / "out" / "r.h5"))
    np.testing.assert_array_equal(back.chain, r.chain)
    np.testing.assert_array_equal(back.accept, r.accept)
    assert back.ndim == 7 and back.wall_time == 1.5 and back.message == "ok"
