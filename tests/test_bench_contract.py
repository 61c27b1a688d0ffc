"""bench.py's output contract, checked on the CPU through its reference arm.

`bench.py --impl reference` times the oracle (the reference's algorithm
restated in C++) on the host cores and prints one JSON line with the same
keys as the GPU arm plus `impl`, `cpu_baseline` and a host-only `e2e`.  A
small grid keeps this to a few seconds.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

REQUIRED = ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
            "scaling", "vs_baseline", "dtype", "data", "config"]


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--size", "65", "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    for k in REQUIRED:
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "node-steps/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["dtype"] == "f64" and d["scaling"] == "weak"
    assert d["config"]["workload"].startswith("mfd_65x65")
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["unit"] == d["unit"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_maps_no_cuda_library():
    """The reference arm runs the oracle only: after one of its instances has
    stepped in the bench process, the process has mapped the oracle's library
    and not the CUDA library of the package."""
    code = (
        "import sys; sys.argv=['bench.py']; sys.path.insert(0, %r)\n"
        "import bench\n"
        "bench._oracle_worker((33, 1, 0, 1))\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('fsgpu' if 'libfsgpu.so' in maps else 'no-fsgpu')\n"
        "print('oracle' if 'libfsoracle.so' in maps else 'no-oracle')\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.split() == ["no-fsgpu", "oracle"], out.stdout
