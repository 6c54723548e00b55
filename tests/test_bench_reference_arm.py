"""CPU: bench.py's reference arm runs the reference's CPU kernel (oracle/_ref)
and maps none of this package's CUDA library, in the bench process or in its
worker processes; its JSON line carries the same `config` as the GPU arm's."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
from forcepho_b200 import synth
# the single-source patch keeps the run short; the code path is the arm's own
bench.make_workload = lambda seed, device_render: synth.make_workload("single", seed=seed)
args = bench.parse()
args.steps, args.warmup = 1, 3
bench.run_reference(args)
maps = open("/proc/self/maps").read()
print(json.dumps({{"libfpho_mapped": "libfpho" in maps,
                  "ref_mapped": "compute_gaussians_kernel" in maps}}))
"""


def test_reference_arm_maps_no_product_library():
    from oracle import oracle as O
    if not O.ref_available(1):
        pytest.skip("reference CPU kernel not built (oracle/_ref)")
    out = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT), "--impl",
                          "reference"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    line, maps = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert set(line["config"]) == {"workload", "pairs_per_eval"}
    assert line["cpu_baseline"]["kind"] == "reference"
    assert maps["libfpho_mapped"] is False


def test_workload_config_is_shared():
    sys.path.insert(0, ROOT)
    import bench
    from forcepho_b200 import synth
    P = synth.make_workload("single", seed=0)
    assert bench.workload_config(P) == {"workload": bench.WORKLOAD,
                                        "pairs_per_eval": int(P.pairs_per_eval)}
