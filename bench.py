#!/usr/bin/env python
"""Benchmark of the proposal-evaluation hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the realistic plain patch (20 Sersic sources, 8 bands x 4
exposures of 128x128 px, 5-Gaussian PSFs, 9 mixture radii: 524,288 pixels x
900 image Gaussians per exposure = 4.72e8 pixel-Gaussian pairs per
evaluation), synthetic and seeded (forcepho_b200.synth, "field20").  A step is
one chi2 + gradient evaluation of one proposal on that patch.  With N GPUs
(torchrun) every rank evaluates its own copy of the patch (independent
patches: weak scaling, no collective on the data path).

Printed JSON (rank 0):
  value      evaluations/s over all ranks, inputs resident in HBM, CUDA-event
             timed per step with an L2 flush between steps (max over ranks);
  e2e        the same through GPUProposer.evaluate_proposal with the proposal
             in pinned host memory and results copied back every step;
  roofline   the pixel-tile kernel: algorithmic FP32 flops (105 per evaluated
             pixel-Gaussian pair) / its CUDA-event time, against the FP32 FMA
             throughput measured live by a probe kernel on the same GPU;
  cpu_baseline  the reference's own CPU kernel (built from its sources into
             oracle/_ref) on all host cores, one evaluation of the same patch.
Further legs on one GPU (each skippable): differentiable (LnLike + leapfrog
in a CUDA graph), multichain (many HMC chains per launch), batched (256
uneven patches in one persistent launch, launch configuration from the batch
autotuner), flux_solve (the fused linear flux solve against the design
matrix + cuBLAS and the host path) and packing (patches packed from a
GPU-resident exposure store against host packing of the same HDF5 store).
The reference arm (--impl reference) times that CPU kernel over K steps.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "chi2+grad evals/s & pix·gauss/s: batched vs plain, 1 B200, rel err ≤1e-6"
FLOPS_PER_PAIR = 105          # 18 (model) + 87 (gradient) FP32 flops, FMA = 2
WORKLOAD = "field20: 20 src, 8 bands x 4 exp x 128x128 px, 5-gauss PSF, 9 radii"
# DRAM bytes (read + write) of one tile-kernel launch on this workload, from an
# ncu capture of one launch of the split tile kernel: the 16 B per pixel of the
# pixel arrays plus the image-Gaussian table, each read once.
TILE_TRAFFIC_BYTES = 12675584
# DRAM bytes of one store_copy launch packing a 471 k-pixel patch (ncu:
# throughput x duration of one launch).
STORE_COPY_TRAFFIC_BYTES = 3833600
# ... and of the one store_copy launch packing the 32 patches of the packing
# leg together (15.07 M pixels; same capture method).
STORE_COPY_BATCH_TRAFFIC_BYTES = 261868000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 1000 on the GPU, 20 for the CPU reference)")
    ap.add_argument("--warmup", type=int, default=None,
                    help="untimed warm-up steps (default 20 on the GPU, 3 for the reference)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--live-cap", type=int, default=None)
    ap.add_argument("--schedule", type=int, default=None, choices=[0, 1],
                    help="0: one CTA per tile; 1: persistent CTAs, costliest tiles first")
    ap.add_argument("--batch-patches", type=int, default=256,
                    help="patches of the batched leg (uneven patches); 0 skips it")
    ap.add_argument("--batch-config", default=None, metavar="VARIANT,LIVE_CAP,CTAS_PER_SM",
                    help="launch configuration of the batched leg (default: the batch "
                         "autotuner's choice)")
    ap.add_argument("--chains", type=int, default=256,
                    help="HMC chains of the multi-chain leg (single-source patch); 0 skips it")
    ap.add_argument("--no-differentiable", action="store_true",
                    help="skip the differentiable-form leg (20-source patch)")
    ap.add_argument("--no-flux", action="store_true",
                    help="skip the flux-solve leg (20-source patch, fixed shapes)")
    ap.add_argument("--packing-patches", type=int, default=32,
                    help="patches packed from the exposure store in the packing leg; 0 skips it")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples SM clock and throttle reasons with nvidia-smi from a thread,
    one query at a time, for as long as the context is open (plus one sample
    on entry and one on exit)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        import threading
        self.idx = gpu_index
        self.lines = []
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._run, daemon=True)

    def _query(self):
        try:
            out = subprocess.run(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                  "--format=csv,noheader,nounits"], capture_output=True,
                                 text=True, timeout=10).stdout
            self.lines.extend(ln for ln in out.splitlines() if ln.strip())
        except (OSError, subprocess.SubprocessError):
            pass

    def _run(self):
        while not self._stop.is_set():
            self._query()
            self._stop.wait(0.05)

    def __enter__(self):
        self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thread.join(timeout=15)
        self._query()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU reference
def cpu_reference_time(P, prop, reps, cores):
    """Seconds per full evaluation (all bands) of the reference CPU kernel,
    bands spread over `cores` spawn worker processes."""
    from oracle import oracle as O
    if not O.ref_available(P.n_sources):
        O.build()
    pool = O.ref_pool(P.n_sources, cores)
    try:
        O.ref_evaluate(P, prop, pool=pool)  # warm-up (loads the module everywhere)
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            O.ref_evaluate(P, prop, pool=pool)
            times.append(time.perf_counter() - t0)
    finally:
        pool.close()
        pool.join()
    return times


def max_over_ranks(x, world, device="cuda"):
    """The largest `x` over the ranks (every rank takes part; NCCL needs a CUDA
    tensor, gloo a CPU one)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(steps, seconds, world):
    """Evaluations per second of the whole job: every rank evaluates `steps`
    patches, the job takes the slowest rank's `seconds`."""
    return world * steps / seconds


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def workload_config(P):
    """The `config` of the JSON line, identical in both arms (run details of
    this implementation go under `run_config`)."""
    return {"workload": WORKLOAD, "pairs_per_eval": int(P.pairs_per_eval)}


def make_workload(seed, device_render):
    from forcepho_b200 import synth
    render = synth.render_model_gpu if device_render else None
    return synth.make_workload("field20", seed=seed, render=render)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    P = make_workload(args.seed, device_render=False)
    prop = P.proposal()
    cores = len(os.sched_getaffinity(0))
    times = cpu_reference_time(P, prop, args.warmup + args.steps, min(cores, P.n_bands))
    t = times[args.warmup:]
    sec = float(np.mean(t))
    value = 1.0 / sec
    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(P),
        "pix_gauss_per_s": P.pairs_per_eval * value,
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": min(cores, P.n_bands),
                         "kind": "reference",
                         "sample": "one full evaluation (8 bands, one band per process) per step"},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def probe_fp32(torch, lib):
    """Measured FP32 FMA (TFLOP/s) and MUFU.EX2 (Gop/s) throughput."""
    dev = torch.cuda.current_device()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    out = torch.zeros(sms * 16, device="cuda")
    s = torch.cuda.current_stream()
    res = {}
    for which, iters, per in ((0, 4096, 32), (1, 1024, 8)):
        blocks, threads = sms * 8, 256
        for rep in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            lib.call("fpho_probe_launch", which, blocks, threads, iters, out.data_ptr(),
                     s.cuda_stream)
            e1.record(s)
            torch.cuda.synchronize()
            rate = blocks * threads * iters * per / (e0.elapsed_time(e1) * 1e-3)
            res[which] = max(res.get(which, 0.0), rate)
    return res[0] / 1e12, res[1] / 1e9


def batched_leg(args, torch, lib, steps):
    """256 uneven patches.  Batched evaluation (one persistent launch
    per step, replayed from a CUDA graph) against the plain form (one
    fpho_evaluate_proposal per patch), both on device-resident buffers."""
    from forcepho_b200 import synth
    from forcepho_b200.batch import PatchBatch
    patches = synth.make_workload("uneven", seed=args.seed + 3, render=synth.render_model_gpu,
                                n_patches=args.batch_patches)
    for P in patches:
        P.return_residual = False
        P.send_to_device()
    # the batch autotuner: tile variant, stage size and persistent-grid cap,
    # timed on this batch (cached by the batch's signature)
    from forcepho_b200.autotune import choose_batch_config
    if args.batch_config:
        v, lc, c = (int(x) for x in args.batch_config.split(","))
        bcfg = {"variant": v, "live_cap": lc, "ctas_per_sm": c}
    else:
        bcfg = choose_batch_config(patches)
    batch = PatchBatch(patches, config=bcfg)
    dprop, chi2, dchi2 = batch.device_buffers()
    s = torch.cuda.current_stream()
    nominal = int(sum(P.pairs_per_eval for P in patches))
    batch.count_pairs(True)
    batch.evaluate_device(dprop, chi2, dchi2)
    torch.cuda.synchronize()
    evaluated = batch.count_pairs(False)
    graph = batch.capture_graph(dprop, chi2, dchi2)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(fn, n):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(n)]
        for e0, e1 in evs:
            flush.zero_()
            e0.record(s)
            fn()
            e1.record(s)
        torch.cuda.synchronize()
        return float(np.sum([a.elapsed_time(b) for a, b in evs])) / n

    for _ in range(3):
        graph.replay()
    ms_batched = timed(graph.replay, steps)
    batch.time_tiles(True)
    tile_ms = []
    for _ in range(min(steps, 10)):
        flush.zero_()
        batch.evaluate_device(dprop, chi2, dchi2)
        tile_ms.append(batch.last_tile_ms())
    batch.time_tiles(False)
    tile_ms = float(np.median(tile_ms))

    # plain: one launch sequence per patch, device buffers per patch
    bufs = []
    for P in patches:
        q = torch.from_numpy(P.proposal().view(np.uint8).copy()).cuda()
        c = torch.zeros(P.n_bands, dtype=torch.float64, device="cuda")
        g = torch.zeros(P.n_bands * P.n_sources * 7, dtype=torch.float32, device="cuda")
        bufs.append((P.device_patch.handle, q, c, g, P.n_sources))

    def plain():
        for h, q, c, g, ns in bufs:
            lib.call("fpho_evaluate_proposal", h, q.data_ptr(), ns, c.data_ptr(), g.data_ptr(),
                     7 * ns, 0, s.cuda_stream)

    for _ in range(2):
        plain()
    ms_plain = timed(plain, max(3, steps // 4))
    n = len(patches)

    # after the timed runs: the batch's outputs (one more graph replay) against
    # the per-patch evaluations the plain loop left in its buffers
    graph.replay()
    torch.cuda.synchronize()
    bc, bg = batch.split_outputs(chi2.cpu().numpy(), dchi2.cpu().numpy())
    chi2_rel, grad_rel = 0.0, 0.0
    for (h, q, c, g, ns), c_b, g_b in zip(bufs, bc, bg):
        c_p = c.cpu().numpy()
        g_p = g.cpu().numpy().reshape(g_b.shape)
        chi2_rel = max(chi2_rel, float(np.max(np.abs(c_b - c_p) / np.abs(c_p))))
        grad_rel = max(grad_rel, float(np.max(np.abs(g_b - g_p)) / max(np.abs(g_p).max(), 1e-30)))
    batch_err = batch.error_word()
    if not (chi2_rel <= 1e-6 and grad_rel <= 1e-5 and batch_err == 0):
        raise RuntimeError(f"batched evaluation differs from the per-patch one: chi2 rel "
                           f"{chi2_rel:.3g}, gradient {grad_rel:.3g} of its largest component, "
                           f"error word {batch_err}")
    out = {"workload": f"uneven: {n} patches, sources U{{1..30}}, bands U{{1..8}}, "
                       "exposures/band U{1..8}, side U[32,200] px",
           "patches": n, "nominal_pairs_per_step": nominal, "evaluated_pairs_per_step": evaluated,
           "work_items": batch.n_work, "persistent_grid": batch.grid,
           "batch_config": dict(batch.config,
                                tile_shape=list(lib.variant_shapes()[batch.config["variant"]])),
           "batched_ms_per_step": ms_batched, "plain_ms_per_step": ms_plain,
           "batched_patch_evals_per_s": n / (ms_batched * 1e-3),
           "plain_patch_evals_per_s": n / (ms_plain * 1e-3),
           "batched_pix_gauss_per_s": nominal / (ms_batched * 1e-3),
           "speedup_batched_vs_plain": ms_plain / ms_batched,
           "roofline": {"kernel": "batch_tiles", "kernel_ms": tile_ms, "bound": "fp32",
                        "achieved": evaluated * FLOPS_PER_PAIR / (tile_ms * 1e-3) / 1e12,
                        "unit": "TFLOP/s"},
           "timing": "CUDA events per step, L2 flushed between steps; batched step replayed "
                     "from a CUDA graph",
           "check_vs_per_patch": {"chi2_max_rel": chi2_rel, "grad_max_rel_of_patch_max": grad_rel,
                                  "what": "after the timed replays: every patch's chi2 and "
                                          "gradient from the batch against its own "
                                          "fpho_evaluate_proposal (asserted: chi2 <= 1e-6, "
                                          "gradient <= 1e-5 of the patch's largest component)"}}
    del graph

    # the batched differentiable form: device-side proposals (splines) and
    # bounded transform for all patches, one batched evaluation, gradient
    # stacking and the leapfrog update, one step per graph replay
    from forcepho_b200.autograd import BatchPosterior, Leapfrog, default_bounds
    lows, highs = zip(*[default_bounds(P.params, P.n_bands) for P in patches])
    bp = BatchPosterior(batch, lows, highs)
    lf = Leapfrog(bp, eps=1e-3, steps_per_graph=1)
    z0 = bp.inverse_transform(np.concatenate([P.params.reshape(-1) for P in patches]))
    p0 = torch.as_tensor(np.random.default_rng(1).standard_normal(bp.ndim), device="cuda")
    lf.set_state(z0, p0)
    lf.run(3)
    ms_leap = timed(lf.graph.replay, steps)

    # the plain drop-in: FastPosterior.lnprob_and_grad per patch (host proposal
    # from the scipy splines, one GPUProposer call per patch, host I/O)
    from forcepho_b200.model import FastPosterior
    from forcepho_b200.proposal import GPUProposer
    from forcepho_b200.sources import Scene
    def dropin_ms(per_source):
        fps = [FastPosterior(GPUProposer(), P,
                             scene=Scene(P.n_sources, P.n_bands, P.table, per_source=per_source),
                             lower=lo, upper=hi) for P, lo, hi in zip(patches, lows, highs)]
        zs = [f.transform.inverse_transform(P.params.reshape(-1)) for f, P in zip(fps, patches)]
        rng = np.random.default_rng(7)

        def dropin():
            for f, z in zip(fps, zs):
                f.lnprob_and_grad(z + 1e-6 * rng.standard_normal(z.shape))

        dropin()
        reps = 2
        t0 = time.perf_counter()
        for _ in range(reps):
            dropin()
        return (time.perf_counter() - t0) / reps * 1e3

    ms_dropin = dropin_ms(None)
    ms_dropin_ps = dropin_ms(True)
    out.update({
        "batched_leapfrog_ms_per_step": ms_leap,
        "batched_leapfrog_patch_evals_per_s": n / (ms_leap * 1e-3),
        "dropin_ms_per_step": ms_dropin,
        "dropin_patch_evals_per_s": n / (ms_dropin * 1e-3),
        "speedup_batched_differentiable_vs_dropin": ms_dropin / ms_leap,
        "dropin": "FastPosterior.lnprob_and_grad per patch: host Scene proposal (scipy "
                  "splines, all sources per call), GPUProposer.evaluate_proposal with host "
                  "I/O; host wall clock",
        "dropin_per_source_ms_per_step": ms_dropin_ps,
        "speedup_batched_differentiable_vs_dropin_per_source": ms_dropin_ps / ms_leap,
        "dropin_per_source": "the same with the proposal built one source at a time, as the "
                             "reference's Galaxy.proposal does",
    })
    del lf
    batch.free()
    for P in patches:
        P.free()
    return out


def multichain_leg(args, torch, steps, n_chains=256):
    """The single-source 64x64 px patch sampled by many HMC chains at once:
    one leapfrog step of every chain per batched launch sequence (graph
    replay), against one chain on the device posterior (graph replay) and the
    plain drop-in FastPosterior.lnprob_and_grad (host proposal, host I/O)."""
    from forcepho_b200 import synth
    from forcepho_b200.autograd import DevicePosterior, Leapfrog, default_bounds
    from forcepho_b200.model import FastPosterior
    from forcepho_b200.proposal import GPUProposer
    from forcepho_b200.sampling import chain_posterior
    from forcepho_b200.sources import Scene
    P = synth.make_workload("single", seed=args.seed, render=synth.render_model_gpu)
    lo, hi = default_bounds(P.params, P.n_bands)
    s = torch.cuda.current_stream()

    def per_replay(graph, n):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(n)]
        for e0, e1 in evs:
            e0.record(s)
            graph.replay()
            e1.record(s)
        torch.cuda.synchronize()
        return float(np.median([a.elapsed_time(b) for a, b in evs]))

    post = chain_posterior(P, n_chains, lo, hi)
    z0 = post.inverse_transform(np.tile(P.params.reshape(-1), n_chains))
    rng = np.random.default_rng(4)
    lf = Leapfrog(post, eps=1e-3, steps_per_graph=1)
    lf.set_state(z0, torch.as_tensor(rng.standard_normal(post.ndim), device="cuda"))
    lf.run(3)
    ms_multi = per_replay(lf.graph, steps)
    del lf
    for c in post.copies:
        c.free()

    P.send_to_device()
    one = DevicePosterior(P, lo, hi)
    lf1 = Leapfrog(one, eps=1e-3, steps_per_graph=1)
    z1 = one.inverse_transform(P.params.reshape(-1))
    lf1.set_state(z1, torch.as_tensor(rng.standard_normal(one.ndim), device="cuda"))
    lf1.run(3)
    ms_one = per_replay(lf1.graph, steps)
    del lf1

    fp = FastPosterior(GPUProposer(), P, scene=Scene(P.n_sources, P.n_bands, P.table),
                       lower=lo, upper=hi)
    z = fp.transform.inverse_transform(P.params.reshape(-1))
    fp.lnprob_and_grad(z)
    n = 50
    t0 = time.perf_counter()
    for _ in range(n):
        fp.lnprob_and_grad(z + 1e-6 * rng.standard_normal(z.shape))
    ms_dropin = (time.perf_counter() - t0) / n * 1e3
    P.free()
    return {"workload": "single: 1 source, 1 band x 1 exposure, 64x64 px (4096 px x 27 "
                        f"image Gaussians), {n_chains} chains",
            "chains": n_chains,
            "multichain_step_ms": ms_multi,
            "multichain_chain_evals_per_s": n_chains / (ms_multi * 1e-3),
            "one_chain_step_ms": ms_one, "one_chain_evals_per_s": 1e3 / ms_one,
            "dropin_ms_per_eval": ms_dropin, "dropin_evals_per_s": 1e3 / ms_dropin,
            "speedup_multichain_vs_dropin": (n_chains / ms_multi) / (1.0 / ms_dropin),
            "timing": "CUDA events per graph replay of one leapfrog step (inputs L2-resident: "
                      "the patch is 64 KB); drop-in: host wall clock"}


def measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool (MEASURED_PEAKS.json beside
    this file), else the earlier pool measurement of 6650 GB/s."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback: earlier measurement on this pool"


def packing_leg(args, torch, n_patches):
    """Patches packed from an exposure store: 8 bands x 4 exposures of
    2048x2048 px in the reference's HDF5 super-pixel layout, circular regions
    of 1.92 arcsec (~128 px across) at random positions.  Device: exposures
    resident in HBM, selection + gather kernels (GPUStorePatch.build_patch:
    exposure finding and pixel packing).  Host: the reference's algorithm
    (StorePatch.build_patch, bit-identical output) on a bounded sample."""
    import shutil
    import tempfile
    from forcepho_b200 import synth
    from forcepho_b200.patches.device_store import DeviceStore, GPUStorePatch
    from forcepho_b200.patches.pixel_patch import StorePatch
    from forcepho_b200.patches.storage import PixelStore
    from forcepho_b200.region import CircularRegion
    d = tempfile.mkdtemp(prefix="fpho_store_")
    try:
        st = synth.make_store(d, n_bands=8, exposures_per_band=4, nside=2048, seed=args.seed,
                              n_sources=20)
        rng = np.random.default_rng(args.seed + 7)
        cosd = np.cos(np.deg2rad(synth.DEC0))
        regions = [CircularRegion(53.16 + rng.uniform(-5, 5) / 3600.0 / cosd,
                                  synth.DEC0 + rng.uniform(-5, 5) / 3600.0, 1.92 / 3600.0)
                   for _ in range(n_patches + 3)]
        t0 = time.perf_counter()
        ds = DeviceStore.from_pixelstore(PixelStore(st["pixelstore"]))
        torch.cuda.synchronize()
        upload_s = time.perf_counter() - t0
        gp = GPUStorePatch(st["pixelstore"], st["metastore"], st["psfstore"], device_store=ds)
        for r in regions[:3]:
            gp.build_patch(r, None, allbands=st["bands"])
        ds.time_gather(True)
        gather_ms, npix = [], []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for r in regions[3:]:
            gp.build_patch(r, None, allbands=st["bands"])
            gather_ms.append(ds.last_gather_ms())
            npix.append(gp.npix)
        torch.cuda.synchronize()
        dev_s = (time.perf_counter() - t0) / n_patches
        hp = StorePatch(st["pixelstore"], st["metastore"], st["psfstore"])
        hp.build_patch(regions[0], None, allbands=st["bands"])          # warm the page cache
        n_host = min(4, n_patches)
        t0 = time.perf_counter()
        for r in regions[3:3 + n_host]:
            hp.build_patch(r, None, allbands=st["bands"])
        host_s = (time.perf_counter() - t0) / n_host
        # all the regions in one count and one gather (GPUStorePatch.build_patches)
        gp.build_patches(regions[3:], None, allbands=st["bands"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        many = gp.build_patches(regions[3:], None, allbands=st["bands"])
        torch.cuda.synchronize()
        many_s = time.perf_counter() - t0
        many_ms = ds.last_gather_ms()
        many_px = sum(q.npix for q in many)
        del many

        # patches ready to evaluate: pixels, 20-source metadata, device handle
        cat = st["catalog"]

        def ready(patch, r):
            patch.build_patch(r, cat, allbands=st["bands"])
            patch.send_to_device()
            patch.free()

        ready(gp, regions[0])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for r in regions[3:]:
            ready(gp, r)
        torch.cuda.synchronize()
        dev_ready_s = (time.perf_counter() - t0) / n_patches

        from forcepho_b200.patches.device_patch import GPUPatchMixin

        class HostStorePatch(StorePatch, GPUPatchMixin):
            pass

        hr = HostStorePatch(st["pixelstore"], st["metastore"], st["psfstore"])
        ready(hr, regions[0])
        t0 = time.perf_counter()
        for r in regions[3:3 + n_host]:
            ready(hr, r)
        torch.cuda.synchronize()
        host_ready_s = (time.perf_counter() - t0) / n_host

        gp.build_patch(regions[2 + n_host], None, allbands=st["bands"])
        gp.pixels_to_host()
        identical = all(np.array_equal(np.asarray(getattr(gp, k)), np.asarray(getattr(hp, k)))
                        for k in ("data", "ierr", "xpix", "ypix", "exposure_start", "exposure_N",
                                  "band_start", "band_N"))
        ds.free()
    finally:
        shutil.rmtree(d, ignore_errors=True)
    peak, peak_src = measured_hbm_gbs()
    g_ms = float(np.median(gather_ms))
    mean_px = float(np.mean(npix))
    achieved = mean_px * 24 / (g_ms * 1e-3) / 1e9
    return {"workload": "store: 8 bands x 4 exposures of 2048x2048 px (8x8 super-pixels, "
                        "1 GiB in HBM), circular regions of 1.92 arcsec, "
                        f"{mean_px:.0f} px per patch",
            "metric": "patches packed/s", "device_patches_per_s": 1.0 / dev_s,
            "host_patches_per_s": 1.0 / host_s, "speedup": host_s / dev_s,
            "batched": {"what": f"{n_patches} patches per GPUStorePatch.build_patches call "
                                "(one count, one gather)",
                        "device_patches_per_s": n_patches / many_s,
                        "gather_ms": many_ms, "pixels": many_px,
                        "achieved_gbs": many_px * 24 / (many_ms * 1e-3) / 1e9,
                        "frac": many_px * 24 / (many_ms * 1e-3) / 1e9 / peak},
            "ready": {"what": "pixels + 20-source metadata (pack_meta) + device patch handle "
                              "with its tile plan (send_to_device), per patch",
                      "device_per_s": 1.0 / dev_ready_s, "host_per_s": 1.0 / host_ready_s,
                      "speedup": host_ready_s / dev_ready_s},
            "host_sample": f"{n_host} patches, StorePatch.build_patch on 1 core: the "
                           "reference's selection and output, HDF5 store in the page cache, "
                           "reading only the selected super-pixels through a memory map (the "
                           "reference reads each exposure whole)",
            "identical_to_host": bool(identical), "store_upload_s": upload_s,
            "roofline": {"bound": "hbm", "kernel": "store_compact + store_copy",
                         "workload": f"{n_patches} patches in one gather "
                                     f"({many_px} pixels)",
                         "kernel_ms": many_ms, "algorithmic_bytes_per_px": 24,
                         "achieved": many_px * 24 / (many_ms * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": many_px * 24 / (many_ms * 1e-3) / 1e9 / peak,
                         "peak_source": peak_src,
                         "traffic": STORE_COPY_BATCH_TRAFFIC_BYTES if n_patches == 32 else None,
                         "traffic_source": "ncu DRAM bytes (throughput x duration) of the "
                                           "32-patch store_copy launch; part of the "
                                           "written output is still in L2 at its end"},
            "single_patch_roofline": {
                "kernel": "store_compact + store_copy", "kernel_ms": g_ms,
                "achieved": achieved, "unit": "GB/s", "frac": achieved / peak,
                "traffic": STORE_COPY_TRAFFIC_BYTES,
                "traffic_source": "ncu DRAM bytes of one store_copy launch of a 471 k-pixel "
                                  "patch (the reads; the outputs stay in L2 during the "
                                  "kernel)"}}


def flux_leg(args, torch, steps):
    """The linear flux solve of the 20 sources of the 20-source patch at
    fixed shapes (forcepho's optimize_fluxes): the fused device solve
    (fpho_patch_optimize_fluxes: per-tile FP64 normal equations without a
    stored design matrix, Cholesky per band) against the design matrix
    written to HBM and the normal equations as FP64 cuBLAS products with a
    batched solve (torch), both on device buffers and CUDA-event timed; and
    the host path as the reference runs it (design matrix copied to the host,
    numpy normal equations and solves), wall clock."""
    from forcepho_b200 import _lib, synth
    from forcepho_b200.fitting import optimize_fluxes
    P = synth.make_workload("field20", seed=args.seed, render=synth.render_model_gpu)
    P.return_residual = False
    P.send_to_device()
    scene = P.set_scene(np.arange(P.n_sources), params=P.truth)
    P.pack_meta(scene)
    P.replace_device_meta_ptrs()
    prop = np.ascontiguousarray(scene.get_proposal())
    ns, nb = len(prop), P.n_bands
    s = torch.cuda.current_stream()
    dprop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    flux = torch.empty((nb, ns), dtype=torch.float64, device="cuda")
    prec = torch.empty((nb, ns, ns), dtype=torch.float64, device="cuda")
    status = torch.zeros(nb, dtype=torch.int32, device="cuda")
    y = torch.as_tensor(P.data, device="cuda", dtype=torch.float64)
    w = torch.as_tensor(P.ierr, device="cuda", dtype=torch.float64)
    cuts = [int(c) for c in np.concatenate([[0], np.cumsum(P.band_N_pix)])]

    def fused():
        _lib.call("fpho_patch_optimize_fluxes", P.device_patch.handle, dprop.data_ptr(), ns,
                  flux.data_ptr(), prec.data_ptr(), status.data_ptr(), s.cuda_stream)

    def unfused():
        X = P.design_matrix_device(prop).to(torch.float64)
        ata = torch.stack([(X[:, a:b] * w[a:b]) @ (X[:, a:b] * w[a:b]).T
                           for a, b in zip(cuts[:-1], cuts[1:])])
        atb = torch.stack([(X[:, a:b] * w[a:b]) @ (y[a:b] * w[a:b])
                           for a, b in zip(cuts[:-1], cuts[1:])])
        return torch.linalg.solve(ata, atb), ata

    def timed(fn, n):
        for _ in range(3):
            fn()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(n)]
        for e0, e1 in evs:
            e0.record(s)
            fn()
            e1.record(s)
        torch.cuda.synchronize()
        return float(np.median([a.elapsed_time(b) for a, b in evs]))

    ms_fused = timed(fused, steps)
    ms_unfused = timed(unfused, steps)
    fl_u, pr_u = unfused()
    torch.cuda.synchronize()
    rel_prec = float((prec - pr_u).abs().max() / pr_u.abs().max())
    rel_flux = float(((flux - fl_u).abs() / fl_u.abs().clamp_min(1e-300)).max())
    optimize_fluxes(P, scene)
    t0 = time.perf_counter()
    n_host = 3
    for _ in range(n_host):
        optimize_fluxes(P, scene)
    host_ms = (time.perf_counter() - t0) / n_host * 1e3
    P.free()
    return {"workload": "field20 flux solve: 20 sources, 8 bands x 4 exposures x 128x128 px, "
                        "fixed shapes",
            "fused_ms": ms_fused, "design_matrix_plus_cublas_ms": ms_unfused,
            "host_reference_path_ms": host_ms, "speedup_vs_design_matrix": ms_unfused / ms_fused,
            "speedup_vs_host": host_ms / ms_fused, "max_rel_diff_precision": rel_prec,
            "max_rel_diff_flux": rel_flux, "status": int(status.sum().item()),
            "timing": "device: CUDA events per call (median); host: wall clock of "
                      "fitting.optimize_fluxes (device design matrix, copied to the host, numpy)"}


def differentiable_leg(args, torch, P, cfg, steps):
    """The 20-source patch through the autograd Function and the
    device posterior, HMC leapfrog steps of 1e-3 in the unconstrained
    coordinates replayed from a CUDA graph, against the plain drop-in
    (FastPosterior.lnprob_and_grad with host proposals and host I/O)."""
    from forcepho_b200.autograd import DevicePosterior, Leapfrog, default_bounds
    from forcepho_b200.model import FastPosterior
    from forcepho_b200.proposal import GPUProposer
    from forcepho_b200.sources import Scene
    s = torch.cuda.current_stream()
    lo, hi = default_bounds(P.params, P.n_bands)
    post = DevicePosterior(P, lo, hi)
    z0 = post.inverse_transform(P.params.reshape(-1))
    p0 = torch.as_tensor(np.random.default_rng(2).standard_normal(post.ndim), device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # one step per replay, L2 flushed between steps
    lf = Leapfrog(post, eps=1e-3, steps_per_graph=1, use_autograd=True)
    lf.set_state(z0, p0)
    lf.run(3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    for e0, e1 in evs:
        flush.zero_()
        e0.record(s)
        lf.graph.replay()
        e1.record(s)
    torch.cuda.synchronize()
    ms_step = float(np.mean([a.elapsed_time(b) for a, b in evs]))

    # the 500-step trajectory back to back (50 steps per graph; L2 stays warm)
    lf50 = Leapfrog(post, eps=1e-3, steps_per_graph=50, use_autograd=True)
    lf50.set_state(z0, p0)
    h0 = float(lf50.hamiltonian())
    lf50.run(50)
    lf50.set_state(z0, p0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    lf50.run(500)
    e1.record(s)
    torch.cuda.synchronize()
    ms_traj = e0.elapsed_time(e1)
    h1 = float(lf50.hamiltonian())
    err = post.ev.error_word()

    def dropin_ms(per_source):
        fp = FastPosterior(GPUProposer(), P,
                           scene=Scene(P.n_sources, P.n_bands, P.table, per_source=per_source),
                           lower=lo, upper=hi)
        z = fp.transform.inverse_transform(P.params.reshape(-1))
        rng = np.random.default_rng(3)
        fp.lnprob_and_grad(z)
        n = 20
        t0 = time.perf_counter()
        for _ in range(n):
            fp.lnprob_and_grad(z + 1e-6 * rng.standard_normal(z.shape))
        return (time.perf_counter() - t0) / n * 1e3

    ms_dropin = dropin_ms(None)
    ms_dropin_ps = dropin_ms(True)
    out = {"workload": "field20 differentiable: 20-source patch, 280 parameters, leapfrog eps 1e-3 in "
                       "unconstrained coordinates",
           "graph_step_ms": ms_step, "graph_evals_per_s": 1e3 / ms_step,
           "trajectory_500_ms": ms_traj, "trajectory_evals_per_s": 500 / (ms_traj * 1e-3),
           "trajectory_dH": h1 - h0, "error_word": err,
           "dropin_ms_per_eval": ms_dropin, "dropin_evals_per_s": 1e3 / ms_dropin,
           "speedup_vs_dropin": ms_dropin / ms_step,
           "dropin_per_source_ms_per_eval": ms_dropin_ps,
           "speedup_vs_dropin_per_source": ms_dropin_ps / ms_step,
           "dropin_per_source": "the same with the proposal built one source at a time, as "
                                "the reference's Galaxy.proposal does",
           "timing": "graph step: CUDA events per replay, L2 flushed between steps; "
                     "trajectory: CUDA events around 10 replays of 50 steps (L2 warm); "
                     "drop-in: host wall clock per FastPosterior.lnprob_and_grad"}
    del lf, lf50
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from forcepho_b200 import _lib
    from forcepho_b200.proposal import GPUProposer
    from forcepho_b200.autotune import apply_config, choose_config

    P = make_workload(args.seed, device_render=True)
    prop = P.proposal()
    P.return_residual = False
    P.send_to_device()
    dp = P.device_patch
    cfg = choose_config(P, variant=args.variant, live_cap=args.live_cap, schedule=args.schedule)
    apply_config(P, cfg)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    dprop = torch.from_numpy(prop.view(np.uint8).copy()).cuda()
    nb, ns = P.n_bands, P.n_sources
    chi2 = torch.zeros(nb, dtype=torch.float64, device="cuda")
    dchi2 = torch.zeros(nb * ns * 7, dtype=torch.float32, device="cuda")

    def step():
        _lib.call("fpho_evaluate_proposal", dp.handle, dprop.data_ptr(), ns, chi2.data_ptr(),
                  dchi2.data_ptr(), 7 * ns, 0, sp)

    # evaluated pairs (after per-tile culling), counted once
    _lib.call("fpho_patch_count_pairs", dp.handle, 1, None)
    step()
    torch.cuda.synchronize()
    import ctypes
    cnt = ctypes.c_longlong()
    _lib.call("fpho_patch_count_pairs", dp.handle, 0, ctypes.byref(cnt))
    evaluated_pairs = int(cnt.value)

    # L2 (126 MB) is flushed between timed steps by writing 256 MB; the flush
    # sits between the step's events, outside the timed intervals.
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for e0, e1 in evs:
            flush.zero_()
            e0.record(stream)
            step()
            e1.record(stream)
        torch.cuda.synchronize()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in evs]
    if world > 1:
        dist.barrier()

    # the dominant kernel alone: events recorded by the library around it
    _lib.call("fpho_patch_time_tiles", dp.handle, 1)
    tms = ctypes.c_float()
    tile_ms = []
    for _ in range(min(args.steps, 50)):
        flush.zero_()
        step()
        _lib.call("fpho_patch_last_tile_ms", dp.handle, ctypes.byref(tms))
        tile_ms.append(tms.value)
    _lib.call("fpho_patch_time_tiles", dp.handle, 0)

    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    ms_per_step = total_ms / args.steps
    value = whole_job_rate(args.steps, total_ms * 1e-3, world)

    # end-to-end through the public API: pinned host proposal -> results on host
    hprop = torch.from_numpy(prop.view(np.uint8).copy()).pin_memory()
    hchi2 = torch.zeros(nb, dtype=torch.float64).pin_memory()
    hdchi2 = torch.zeros(nb * ns * 7, dtype=torch.float32).pin_memory()

    def e2e_step():
        _lib.call("fpho_evaluate_proposal", dp.handle, hprop.data_ptr(), ns, hchi2.data_ptr(),
                  hdchi2.data_ptr(), 7 * ns, _lib.FPHO_IO_HOST, sp)

    for _ in range(args.warmup):
        e2e_step()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = whole_job_rate(args.steps, e2e_s, world)

    fp32_tflops, ex2_gops = probe_fp32(torch, _lib)
    tile_s = float(np.mean(tile_ms)) * 1e-3
    achieved = evaluated_pairs * FLOPS_PER_PAIR / tile_s / 1e12
    sfu = evaluated_pairs * 2 / tile_s / 1e9

    # the further legs run in single-GPU runs only (a multi-GPU run measures
    # the patch-parallel evaluation and holds every GPU while it runs)
    differentiable = None
    if world == 1 and not args.no_differentiable:
        differentiable = differentiable_leg(args, torch, P, cfg, steps=max(3, min(args.steps, 50)))

    multichain = None
    if world == 1 and args.chains > 0:
        multichain = multichain_leg(args, torch, steps=max(3, min(args.steps, 50)),
                                    n_chains=args.chains)

    batched = None
    if world == 1 and args.batch_patches > 0:
        batched = batched_leg(args, torch, _lib, steps=max(3, min(args.steps, 50)))
        rb = batched["roofline"]
        rb.update({"peak": fp32_tflops, "frac": rb["achieved"] / fp32_tflops,
                   "peak_source": "measured live: packed FP32 FMA probe kernel"})

    flux = None
    if rank == 0 and world == 1 and not args.no_flux:
        flux = flux_leg(args, torch, steps=max(3, min(args.steps, 50)))

    packing = None
    if rank == 0 and world == 1 and args.packing_patches > 0:
        packing = packing_leg(args, torch, args.packing_patches)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = len(os.sched_getaffinity(0))
        use = min(cores, nb)
        times = cpu_reference_time(P, prop, 5, use)
        one = cpu_reference_time(P, prop, 1, 1)
        cpu = {"value": 1.0 / float(np.median(times)), "unit": "evals/s", "cores": use,
               "kind": "reference",
               "single_core_evals_per_s": 1.0 / float(one[0]),
               "cpu_model": _cpu_model(),
               "sample": "median of 5 full evaluations of the same patch after one warm-up "
                         f"(8 bands, one band per process on {use} of {cores} host cores); "
                         "single core: one full evaluation, bands in turn"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": workload_config(P),
            "run_config": {"evaluated_pairs": evaluated_pairs, "l2": "flushed between steps",
                           "tile_variant": cfg["variant"],
                           "tile_shape": dict(zip(("threads", "pixels_per_tile",
                                                   "warps_sharing_gaussians"),
                                                  _lib.variant_shapes()[cfg["variant"]])),
                           "live_cap": cfg["live_cap"], "schedule": cfg.get("schedule", 0),
                           "parallelism": f"patch-parallel x{world}"},
            "pix_gauss_per_s": P.pairs_per_eval * value,
            "evaluated_pix_gauss_per_s": evaluated_pairs * value,
            "e2e": {"value": e2e_value, "unit": "evals/s",
                    "h2d_bytes_per_step": int(prop.nbytes),
                    "d2h_bytes_per_step": int(nb * 8 + nb * ns * 7 * 4 + 4)},
            # per evaluation: prepare_evaluation (image Gaussians, tile order,
            # error word), the tile kernel and reduce_bands
            "gpu_launches": 3 * args.steps,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_tflops,
                         "unit": "TFLOP/s", "frac": achieved / fp32_tflops,
                         "traffic": TILE_TRAFFIC_BYTES,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           "of one launch",
                         "peak_source": "measured live: packed FP32 FMA probe kernel",
                         "kernel": ("split_kernel_dyn" if _lib.variant_shapes()[cfg["variant"]][2]
                                    else "tile_kernel_dyn") if cfg.get("schedule", 0) == 1 else
                                   ("split_kernel" if _lib.variant_shapes()[cfg["variant"]][2]
                                    else "tile_kernel"),
                         "kernel_ms": tile_s * 1e3,
                         "sfu_gops": sfu, "sfu_peak_gops": ex2_gops, "sfu_frac": sfu / ex2_gops},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "differentiable": differentiable,
            "multichain": multichain,
            "batched": batched,
            "flux_solve": flux,
            "packing": packing,
        }
        print(json.dumps(line), flush=True)
    P.free()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    ref = args.impl == "reference"
    if args.steps is None:
        args.steps = 20 if ref else 1000
    if args.warmup is None:
        args.warmup = 3 if ref else 20
    args.warmup = max(args.warmup, 3)
    if ref:
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
