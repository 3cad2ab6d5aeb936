"""bench.py's reference arm on a tiny mesh (CPU only): one JSON line with the
contract's keys, the CPU restatement timed on the host cores."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--mesh", "12,4,4",
                          "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, env={**os.environ, "WORLD_SIZE": "1", "RANK": "0"})
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "MG cycles/s" and d["unit"] == "cycles/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 3
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "cycles/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "12x4x4" in d["config"]["workload"]


def test_other_ranks_of_the_reference_arm_exit_quietly():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--mesh", "12,4,4",
                          "--steps", "1", "--warmup", "3"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, env={**os.environ, "WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]


def test_product_arm_refuses_to_run_without_a_gpu():
    # no CPU fallback: without a CUDA device the product arm stops loudly
    import torch
    if torch.cuda.is_available():
        return
    for extra in ([], ["--upwind"], ["--rans"]):
        out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--mesh", "12,4,4", "--steps", "1",
                              "--warmup", "3", *extra], capture_output=True, text=True, timeout=600, cwd=ROOT)
        assert out.returncode != 0
        assert "no CPU fallback" in out.stderr + out.stdout


def test_reference_arm_does_not_load_the_cuda_library():
    # the CPU arm fills its controls from the host library: the product's
    # CUDA library must not be mapped into its process
    code = ("import sys, bench; sys.argv = ['bench.py', '--impl', 'reference', '--mesh', '8,4,4', '--steps', '1', "
            "'--warmup', '3']; bench.main(); maps = open('/proc/self/maps').read(); "
            "print('GPULIB' if 'libflite_gpu.so' in maps else 'NOGPULIB')")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT,
                         env={**os.environ, "WORLD_SIZE": "1", "RANK": "0"})
    assert out.returncode == 0, out.stderr[-2000:]
    assert "NOGPULIB" in out.stdout
