"""Many patches evaluated by one persistent launch.

The reference evaluates one patch per kernel launch and runs many patches by
giving each MPI child its own patch (forcepho/dispatcher.py).  On a B200 one
small patch cannot fill 148 SMs, so :class:`PatchBatch` evaluates a list of
patches together: one launch builds all image Gaussians, one persistent
launch walks a cost-sorted (patch, tile) work list, one launch reduces every
(patch, band).  ``capture_graph`` records that sequence as a CUDA graph for
replay in a sampler loop.
"""

import ctypes

import numpy as np

from . import _lib
from .kernel_limits import NPARAMS
from .proposal import source_struct_dtype

__all__ = ["PatchBatch", "batch_variants"]


def batch_variants():
    """The tile variants that have a batched kernel (fpho_batch_variants)."""
    out = (ctypes.c_int * 16)()
    n = _lib.lib.fpho_batch_variants(out, 16)
    return [out[i] for i in range(min(n, 16)) if out[i] >= 0]


class PatchBatch:
    """A batch over patches that are already on the device (``send_to_device``).

    Parameters
    ----------
    patches : list of patch objects with a ``device_patch`` (DevicePatch)
    live_cap : image-Gaussian records per shared-memory stage
    variant : tile variant of the batched kernel (one of :func:`batch_variants`;
        None: the default, 64 threads x 8 pixels)
    ctas_per_sm : cap on the persistent grid's resident CTAs per SM (0: none)
    config : a dict from :func:`forcepho_b200.autotune.choose_batch_config`
        (``variant``, ``live_cap``, ``ctas_per_sm``), overriding the above
    """

    def __init__(self, patches, live_cap=128, stream=None, variant=None, ctas_per_sm=0,
                 config=None):
        if config is not None:
            variant = config.get("variant", variant)
            live_cap = config.get("live_cap", live_cap)
            ctas_per_sm = config.get("ctas_per_sm", ctas_per_sm)
        self.patches = list(patches)
        handles = (ctypes.c_void_p * len(self.patches))(
            *[p.device_patch.handle for p in self.patches])
        h = ctypes.c_void_p()
        _lib.call("fpho_batch_create_config", handles, len(self.patches),
                  -1 if variant is None else int(variant), int(live_cap), int(ctas_per_sm),
                  stream, ctypes.byref(h))
        self.handle = h.value
        cfg = (ctypes.c_int * 4)()
        _lib.call("fpho_batch_config", self.handle, cfg)
        self.config = {"variant": cfg[0], "live_cap": cfg[1], "ctas_per_sm": cfg[2]}
        info = (ctypes.c_int64 * 7)()
        _lib.call("fpho_batch_info", self.handle, info)
        self.n_sources_total, self.n_bands_total, self.n_dchi2 = info[1], info[2], info[3]
        self.n_work, self.grid, self.n_exposures = info[4], info[5], info[6]
        self.n_bands = [p.n_bands for p in self.patches]
        self.n_sources = [p.n_sources for p in self.patches]

    # -------------------------------------------------------------- host I/O
    def pack_proposals(self, proposals):
        """Concatenate one ``source_struct_dtype`` array per patch."""
        for p, q in zip(self.patches, proposals):
            if len(q) != p.n_sources:
                raise ValueError("proposal length does not match its patch")
        return np.ascontiguousarray(np.concatenate(proposals), dtype=source_struct_dtype)

    def split_outputs(self, chi2, dchi2):
        """Per-patch (chi2 (n_bands,), dchi2 (n_bands, n_sources, 7)) lists."""
        out_c, out_g, i, j = [], [], 0, 0
        for nb, ns in zip(self.n_bands, self.n_sources):
            out_c.append(chi2[i:i + nb])
            out_g.append(dchi2[j:j + nb * ns * NPARAMS].reshape(nb, ns, NPARAMS))
            i += nb
            j += nb * ns * NPARAMS
        return out_c, out_g

    def evaluate(self, proposals):
        """Evaluate one proposal per patch (host arrays in, host arrays out)."""
        props = self.pack_proposals(proposals)
        chi2 = np.empty(self.n_bands_total, dtype=np.float64)
        dchi2 = np.empty(self.n_dchi2, dtype=np.float32)
        _lib.call("fpho_batch_evaluate", self.handle, props.ctypes.data, chi2.ctypes.data,
                  dchi2.ctypes.data, _lib.FPHO_IO_HOST, None)
        return self.split_outputs(chi2, dchi2)

    # -------------------------------------------------------------- device I/O
    def device_buffers(self, proposals=None):
        """torch device tensors (proposal bytes, chi2, dchi2) for device-resident use."""
        import torch
        if proposals is None:
            proposals = [p.proposal() for p in self.patches]
        props = self.pack_proposals(proposals)
        dprop = torch.from_numpy(props.view(np.uint8).copy()).cuda()
        chi2 = torch.zeros(self.n_bands_total, dtype=torch.float64, device="cuda")
        dchi2 = torch.zeros(self.n_dchi2, dtype=torch.float32, device="cuda")
        return dprop, chi2, dchi2

    def evaluate_device(self, dprop, chi2, dchi2, stream=None):
        """Enqueue an evaluation on device buffers (no synchronization)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _lib.call("fpho_batch_evaluate", self.handle, dprop.data_ptr(), chi2.data_ptr(),
                  dchi2.data_ptr(), 0, s)

    def capture_graph(self, dprop, chi2, dchi2):
        """A torch CUDAGraph replaying one batched evaluation on these buffers."""
        import torch
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.evaluate_device(dprop, chi2, dchi2, s.cuda_stream)  # warm-up outside capture
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.evaluate_device(dprop, chi2, dchi2)
        return g

    def time_tiles(self, enable=True):
        """Record CUDA events around the persistent tile launch."""
        _lib.call("fpho_batch_time_tiles", self.handle, int(enable))

    def last_tile_ms(self):
        """Milliseconds of the last timed tile launch (synchronizes on it)."""
        t = ctypes.c_float()
        _lib.call("fpho_batch_last_tile_ms", self.handle, ctypes.byref(t))
        return float(t.value)

    def error_word(self):
        """The batched kernels' error word of the last evaluation (0 = none)."""
        w = ctypes.c_int()
        _lib.call("fpho_batch_error_word", self.handle, ctypes.byref(w))
        return w.value

    def count_pairs(self, enable=True):
        c = ctypes.c_longlong()
        _lib.call("fpho_batch_count_pairs", self.handle, int(enable), ctypes.byref(c))
        return int(c.value)

    def free(self):
        if getattr(self, "handle", None):
            _lib.lib.fpho_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
