"""GPU: patches packed on the device from the exposure store.

  * the select+gather kernels against oracle/packing.py, bit for bit, on
    random stores: circles inside, across the edge of and around the whole
    image, a circle that misses (0 super-pixels), RA/Dec boxes, background
    offsets, the S/N cap, super-pixels of 8 and 4, non-square images;
  * GPUStorePatch.build_patch against the reference's own StorePatch output
    (tests/golden/packing_store.npz, made by make_packing_golden.py);
  * a patch packed on the device evaluates bit-identically to the same patch
    packed on the host;
  * the data/residual swap of the reference's tests/cswap_test.py:83-110 on
    the reference's test image as its FITSPatch packs it
    (tests/golden/packing_fits.npz);
  * argument errors are reported, not faulted.
"""
import hashlib
import os

import numpy as np
import pytest

from oracle import packing as OP

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def _cases():
    import sys
    sys.path.insert(0, GOLDEN)
    import make_packing_golden as G
    return G


def _random_store(nx, ny, s, n_exp, seed):
    rng = np.random.default_rng(seed)
    sps = []
    for _ in range(n_exp):
        sp = rng.normal(0, 1, (nx // s, ny // s, 2 * s * s)).astype(np.float32)
        sp[..., s * s:] = np.abs(sp[..., s * s:]) * 5
        sp[..., s * s:][rng.uniform(size=sp[..., s * s:].shape) < 0.05] = 0.0
        sp[..., :s * s][rng.uniform(size=sp[..., :s * s].shape) < 0.01] = 40.0
        sps.append(sp)
    return sps


def _rect_params(rng, nx, ny):
    from forcepho_b200 import synth
    from forcepho_b200.region import RectangularRegion
    from forcepho_b200.wcs import TanWCS
    w = TanWCS(synth.store_header("F200W", (nx, ny), (53.1, -27.8),
                                  (nx / 2 + rng.uniform(-5, 5), ny / 2 + rng.uniform(-5, 5)),
                                  rng.uniform(-30, 30)))
    ra, dec = w.pixel_to_world_values(rng.uniform(0.2, 0.8) * nx, rng.uniform(0.2, 0.8) * ny)
    half = rng.uniform(0.5, 4.0) / 3600.0
    return RectangularRegion(ra - half, ra + half * 1.3, dec - half * 0.7, dec + half).device_params(w)


@pytest.mark.parametrize("nx,ny,s", [(512, 384, 8), (256, 256, 4), (64, 136, 8), (96, 72, 3)])
def test_gather_matches_oracle(nx, ny, s):
    from forcepho_b200.patches.device_store import DeviceStore, REGION_DTYPE
    rng = np.random.default_rng(nx + ny + s)
    sps = _random_store(nx, ny, s, 5, seed=s)
    st = DeviceStore((nx, ny), s, max_exposures=5)
    for sp in sps:
        st.add(sp)
    regions = [
        (1, [nx * 0.4, ny * 0.6, (0.2 * min(nx, ny)) ** 2]),         # inside
        (1, [-3.5, ny * 0.5, (0.3 * ny) ** 2]),                      # across the edge
        (1, [nx / 2, ny / 2, float(nx * nx + ny * ny)]),             # the whole image
        (1, [-10 * nx, -10 * ny, 25.0]),                             # misses: 0 super-pixels
        _rect_params(rng, nx, ny),
    ]
    order = [3, 0, 4, 1, 2]
    recs = np.zeros(len(order), dtype=REGION_DTYPE)
    for i, e in enumerate(order):
        recs[i]["kind"] = regions[e][0]
        recs[i]["p"][:len(regions[e][1])] = regions[e][1]
    counts = st.count(order, recs)
    assert counts[0] == 0 and counts[4] == (nx // s) * (ny // s)
    for bg, max_snr in ((None, None), (rng.normal(0, 0.1, len(order)), 30.0)):
        pix, start, n = st.gather(order, recs, background=bg, max_snr=max_snr)
        want = OP.pack([sps[e] for e in order], [regions[e] for e in order], background=bg,
                       max_snr=max_snr)
        np.testing.assert_array_equal(n, want["exposure_N"])
        np.testing.assert_array_equal(start, want["exposure_start"])
        np.testing.assert_array_equal(n, counts * s * s)
        for k, t in zip(("data", "ierr", "xpix", "ypix"), pix):
            np.testing.assert_array_equal(t.cpu().numpy(), want[k], err_msg=k)
    st.free()


def test_gather_random_small_circles():
    """Many small circles: the chunk-level skip of the count and compact
    kernels (chunks of 1024 super-pixels that start and end mid-row here,
    48 super-pixels per row) must not change the selection."""
    from forcepho_b200.patches.device_store import DeviceStore, REGION_DTYPE
    nx, ny, s = 512, 384, 8
    rng = np.random.default_rng(17)
    sps = _random_store(nx, ny, s, 2, seed=5)
    st = DeviceStore((nx, ny), s, max_exposures=2)
    for sp in sps:
        st.add(sp)
    n = 40
    order = rng.integers(0, 2, n)
    regs = [(1, [rng.uniform(-20, nx + 20), rng.uniform(-20, ny + 20),
                 rng.uniform(1.0, 60.0) ** 2]) for _ in range(n)]
    recs = np.zeros(n, dtype=REGION_DTYPE)
    recs["kind"] = 1
    recs["p"][:, :3] = [r[1] for r in regs]
    pix, start, cnt = st.gather(order, recs)
    want = OP.pack([sps[e] for e in order], regs)
    np.testing.assert_array_equal(cnt, want["exposure_N"])
    for k, t in zip(("data", "ierr", "xpix", "ypix"), pix):
        np.testing.assert_array_equal(t.cpu().numpy(), want[k], err_msg=k)
    st.free()


@pytest.fixture(scope="module")
def store(tmp_path_factory):
    from forcepho_b200 import synth
    G = _cases()
    return synth.make_store(str(tmp_path_factory.mktemp("gstore")), seed=G.STORE_SEED,
                            **G.STORE_KW)


def _region(kind, args):
    from forcepho_b200.region import CircularRegion, RectangularRegion
    return CircularRegion(*args) if kind == "circle" else RectangularRegion(*args)


def test_gpu_store_patch_matches_reference(store):
    from forcepho_b200.patches.device_store import DeviceStore, GPUStorePatch
    from forcepho_b200.patches.storage import PixelStore
    G = _cases()
    gold = np.load(os.path.join(GOLDEN, "packing_store.npz"))
    dstore = DeviceStore.from_pixelstore(PixelStore(store["pixelstore"]))
    for name, kind, args, tweak, max_snr in G.STORE_CASES:
        p = GPUStorePatch(store["pixelstore"], store["metastore"], store["psfstore"],
                          device_store=dstore)
        p.max_snr = max_snr
        p.build_patch(_region(kind, args), store["catalog"], allbands=store["bands"],
                      tweak_background=tweak)
        assert list(p.epaths) == [str(e) for e in gold[f"{name}/epaths"]]
        p.pixels_to_host()
        for k in ("data", "ierr", "xpix", "ypix"):
            assert _digest(getattr(p, k)) == str(gold[f"{name}/{k}_sha256"]), (name, k)
        for k in ("exposure_start", "exposure_N", "band_start", "band_N", "D", "CW", "crpix",
                  "crval", "G", "psfgauss_start"):
            np.testing.assert_array_equal(np.asarray(getattr(p, k)), gold[f"{name}/{k}"],
                                          err_msg=f"{name}/{k}")
        p.send_to_device()                 # with host copies present: still the device arrays
        np.testing.assert_array_equal(p.retrieve_array("data"), p.data)
        p.free()
    dstore.free()


def test_device_packed_patch_evaluates_like_host_packed(store):
    from forcepho_b200.patches.device_store import GPUStorePatch
    from forcepho_b200.patches.pixel_patch import StorePatch
    from forcepho_b200.proposal import GPUProposer
    G = _cases()
    name, kind, args, tweak, max_snr = G.STORE_CASES[1]
    from forcepho_b200.patches.device_patch import GPUPatchMixin

    class HostStorePatch(StorePatch, GPUPatchMixin):   # host packing, as the reference's patchers
        pass

    out = []
    for cls in (HostStorePatch, GPUStorePatch):
        p = cls(store["pixelstore"], store["metastore"], store["psfstore"])
        p.max_snr = max_snr
        p.build_patch(_region(kind, args), store["catalog"], allbands=store["bands"],
                      tweak_background=tweak)
        p.send_to_device()
        prop = p.scene.get_proposal()
        out.append(GPUProposer().evaluate_proposal(prop, patch=p))
        p.free()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert np.all(np.isfinite(out[0][0])) and np.any(out[0][1] != 0)


def _fits_patch():
    """The reference's test image as its FITSPatch packed it, with the GPU
    mix-in (cswap_test.py's Patcher)."""
    from forcepho_b200.patches.device_patch import GPUPatchMixin
    from forcepho_b200.patches.patch import PSF_COLS, PSF_DTYPE, PatchBase
    from forcepho_b200.sources import Scene, default_table

    class Patcher(PatchBase, GPUPatchMixin):
        pass

    g = np.load(os.path.join(GOLDEN, "packing_fits.npz"))
    p = Patcher(return_residual=True)
    for k in ("data", "ierr", "xpix", "ypix", "exposure_start", "exposure_N", "band_start",
              "band_N", "D", "CW", "crpix", "crval", "G", "rad2", "n_psf_per_source",
              "psfgauss_start"):
        setattr(p, k, np.array(g[k]))
    ps = np.zeros(len(g["psfgauss"]), dtype=PSF_DTYPE)
    for i, c in enumerate(PSF_COLS + ["sersic_bin"]):
        ps[c] = g["psfgauss"][:, i]
    p.psfgauss = ps
    p.n_sources, p.n_radii = 1, len(g["rad2"])
    cat = g["catalog"][0]                     # ra, dec, q, pa, sersic, rhalf, CLEAR
    params = np.array([[cat[6], cat[0], cat[1], cat[2], cat[3], cat[4], cat[5]]])
    params[0, 1:3] -= g["reference_coordinates"]
    return p, Scene(1, 1, default_table(), params=params)


def test_cswap_on_reference_test_image():
    """tests/cswap_test.py:59-110 of the reference: evaluate, swap the device
    residual into the data, evaluate again -> data - 2 model."""
    from oracle import oracle as O
    from forcepho_b200.proposal import GPUProposer
    patcher, scene = _fits_patch()
    proposer = GPUProposer()
    patcher.send_to_device()
    proposal = scene.get_proposal()
    chi, dchi_dp, residual = proposer.evaluate_proposal(proposal, patch=patcher, unpack=False)
    c32, _ = O.oracle_evaluate(patcher, proposal, precision="f32")
    np.testing.assert_allclose(chi, c32, rtol=1e-6)
    residual_original = residual
    data_original = patcher.data.copy()
    patcher.swap_on_device()
    data_postswap = patcher.retrieve_array("data")
    residual_postswap = patcher.retrieve_array("residual")
    assert np.allclose(residual_original, data_postswap)
    assert np.allclose(data_original, residual_postswap)
    chi, dchi_dp, residual_new = proposer.evaluate_proposal(proposal, patch=patcher, unpack=False)
    model = data_original - residual_original
    assert np.allclose(residual_new, data_original - 2 * model)
    assert np.abs(model).max() > 1e-3          # the galaxy is there
    patcher.free()


def test_store_argument_errors():
    from forcepho_b200 import _lib
    from forcepho_b200.patches.device_store import DeviceStore, REGION_DTYPE
    with pytest.raises(_lib.FphoError, match="INVALID"):
        DeviceStore((100, 64), 8, 1)              # 100 is not a multiple of 8
    st = DeviceStore((64, 64), 8, max_exposures=1)
    st.add(np.zeros((8, 8, 128), dtype=np.float32))
    with pytest.raises(_lib.FphoError, match="LIMIT"):
        st.add(np.zeros((8, 8, 128), dtype=np.float32))
    with pytest.raises(ValueError):
        DeviceStore((64, 64), 8, 2).add(np.zeros((8, 4, 128), dtype=np.float32))
    rec = np.zeros(1, dtype=REGION_DTYPE)
    rec["kind"], rec["p"][0, :3] = 1, [32.0, 32.0, 400.0]
    with pytest.raises(_lib.FphoError, match="INVALID"):
        st.count([1], rec)                        # no exposure 1
    bad = rec.copy()
    bad["kind"] = 7
    with pytest.raises(_lib.FphoError, match="INVALID"):
        st.count([0], bad)
    with pytest.raises(_lib.FphoError, match="LIMIT"):
        st.gather([0], rec, npix=64)              # the selection has more pixels
    assert st.count([0], rec)[0] > 1
    st.free()


def test_build_patches_matches_one_at_a_time(store):
    """GPUStorePatch.build_patches (one count and one gather for all the
    regions) gives each patch the arrays build_patch gives it alone."""
    from forcepho_b200.patches.device_store import DeviceStore, GPUStorePatch
    from forcepho_b200.patches.storage import PixelStore
    from forcepho_b200.region import CircularRegion
    G = _cases()
    ds = DeviceStore.from_pixelstore(PixelStore(store["pixelstore"]))
    gp = GPUStorePatch(store["pixelstore"], store["metastore"], store["psfstore"],
                       device_store=ds)
    gp.max_snr = 100.0
    rng = np.random.default_rng(4)
    regions = [CircularRegion(53.16 + rng.uniform(-2, 2) / 3600, -27.78 + rng.uniform(-2, 2) / 3600,
                              rng.uniform(1.0, 3.0) / 3600) for _ in range(6)]
    regions.append(_region(*G.STORE_CASES[2][1:3]))           # an RA/Dec box
    cats = [store["catalog"][: 1 + i % 4] for i in range(len(regions))]
    many = gp.build_patches(regions, cats, allbands=store["bands"], tweak_background="BKG")
    for region, cat, q in zip(regions, cats, many):
        gp.build_patch(region, cat, allbands=store["bands"], tweak_background="BKG")
        assert list(q.epaths) == list(gp.epaths)
        for k in ("data", "ierr", "xpix", "ypix"):
            np.testing.assert_array_equal(q.pixels[k].cpu().numpy(), gp.pixels[k].cpu().numpy())
        for k in ("exposure_start", "exposure_N", "band_start", "band_N", "D", "CW", "crpix",
                  "crval", "G", "psfgauss_start", "n_psf_per_source"):
            np.testing.assert_array_equal(np.asarray(getattr(q, k)), np.asarray(getattr(gp, k)),
                                          err_msg=k)
    q = many[0]
    q.send_to_device()                                        # a batch-packed patch evaluates
    from forcepho_b200.proposal import GPUProposer
    chi2, dchi2 = GPUProposer().evaluate_proposal(q.scene.get_proposal(), patch=q)
    assert np.all(np.isfinite(chi2))
    q.free()
    ds.free()


def test_gather_unaligned_outputs():
    """Output arrays that are not 16-byte aligned take the one-pixel-per-thread
    copy; the result is the same as the oracle's."""
    import ctypes
    import torch
    from forcepho_b200 import _lib
    from forcepho_b200.patches.device_store import DeviceStore, REGION_DTYPE
    nx, ny, s = 128, 96, 8
    sps = _random_store(nx, ny, s, 2, seed=9)
    st = DeviceStore((nx, ny), s, max_exposures=2)
    for sp in sps:
        st.add(sp)
    regs = [(1, [40.5, 50.25, 30.0 ** 2]), (1, [100.0, 10.0, 25.0 ** 2])]
    recs = np.zeros(2, dtype=REGION_DTYPE)
    recs["kind"] = 1
    recs["p"][:, :3] = [r[1] for r in regs]
    want = OP.pack(sps, regs, max_snr=30.0)
    npix = int(want["exposure_N"].sum())
    bufs = [torch.zeros(npix + 1, dtype=torch.float32, device="cuda") for _ in range(4)]
    start = np.zeros(2, np.int32)
    n = np.zeros(2, np.int32)
    idx = np.arange(2, dtype=np.int32)
    _lib.call("fpho_store_gather", st.handle, 2, idx.ctypes.data, recs.ctypes.data, None,
              ctypes.c_float(30.0), *[b.data_ptr() + 4 for b in bufs], npix, start.ctypes.data,
              n.ctypes.data, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(n, want["exposure_N"])
    for k, b in zip(("data", "ierr", "xpix", "ypix"), bufs):
        np.testing.assert_array_equal(b[1:].cpu().numpy(), want[k], err_msg=k)
        assert float(b[0]) == 0.0                 # nothing written before the output
    st.free()


def test_fixed_sources_on_a_store_patch(store):
    """The reference's fixed-source flow on a patch packed on the device:
    subtract_fixed(fixed, active) leaves data - model(fixed) on the device, so
    evaluating the active scene then gives the joint residual of all sources;
    design_matrix and optimize_fluxes run on it (device_patch.py:113-238,
    fitting.py:597-627)."""
    from forcepho_b200.fitting import optimize_fluxes
    from forcepho_b200.patches.device_store import GPUStorePatch
    G = _cases()
    region = _region(*G.STORE_CASES[0][1:3])
    cat = store["catalog"]
    fixed, active = cat[:2], cat[2:]

    def patcher():
        p = GPUStorePatch(store["pixelstore"], store["metastore"], store["psfstore"],
                          return_residual=True)
        p.build_patch(region, None, allbands=store["bands"])
        return p

    joint = patcher()
    joint.pack_meta(joint.set_scene(cat))
    joint.send_to_device()
    _, _, r_joint = joint.get_proposer().evaluate_proposal(joint.scene.get_proposal(),
                                                           patch=joint, unpack=False)
    data = joint.retrieve_array("data")
    joint.free()

    seq = patcher()
    proposer, scene = seq.subtract_fixed(fixed, active=active)
    _, _, r_seq = proposer.evaluate_proposal(scene.get_proposal(), patch=seq, unpack=False)
    scale = np.abs(data - r_joint).max()
    assert scale > 0
    # the subtraction rounds in the data's precision: the two residuals agree
    # to the model scale plus a few float ulps of the data at each pixel
    tol = 1e-4 * scale + 4 * np.finfo(np.float32).eps * np.abs(data)
    assert np.all(np.abs(r_seq - r_joint) <= tol), float(np.max(np.abs(r_seq - r_joint) - tol))
    Xes, ys = seq.design_matrix(active)
    assert len(Xes) == len(store["bands"]) and Xes[0].shape[0] == len(active)
    fluxes, precisions = optimize_fluxes(seq, active)
    assert np.all(np.isfinite(np.asarray(fluxes, dtype=float)))
    seq.free()


def test_gpu_store_patch_with_sip_headers(tmp_path):
    """Exposures whose headers carry SIP distortion: the device packing (circle
    centre and radius mapped by the SIP-aware WCS on the host) equals the host
    StorePatch's; RA/Dec boxes, which the kernel maps with TAN alone, are
    refused for them."""
    from forcepho_b200 import synth
    from forcepho_b200.patches.device_store import GPUStorePatch
    from forcepho_b200.patches.pixel_patch import StorePatch
    from forcepho_b200.region import CircularRegion, RectangularRegion
    st = synth.make_store(str(tmp_path), seed=5, sip=True, n_bands=2, exposures_per_band=2)
    region = CircularRegion(53.16, -27.78, 2.5 / 3600)
    host = StorePatch(st["pixelstore"], st["metastore"], st["psfstore"])
    host.build_patch(region, st["catalog"], allbands=st["bands"])
    dev = GPUStorePatch(st["pixelstore"], st["metastore"], st["psfstore"])
    dev.build_patch(region, st["catalog"], allbands=st["bands"])
    assert list(dev.epaths) == list(host.epaths)
    for k in ("data", "ierr", "xpix", "ypix"):
        np.testing.assert_array_equal(dev.pixels[k].cpu().numpy(), getattr(host, k), err_msg=k)
    np.testing.assert_array_equal(dev.CW, host.CW)
    with pytest.raises(NotImplementedError):
        dev.build_patch(RectangularRegion(53.159, 53.161, -27.781, -27.779), None,
                        allbands=st["bands"])
