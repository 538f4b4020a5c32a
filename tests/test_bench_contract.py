"""bench.py's reference arm (CPU only): one JSON line with the driver's keys.

The reference arm times the reference algorithm's CPU form (the oracle's BLAS
restatement) on the host cores; it must print the same metric and unit as the
GPU arm, ``impl: reference``, a ``cpu_baseline`` describing the run and an
``e2e`` block with no host<->device bytes.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    # at the small size S: the default size builds a 24.7 GB table on the host
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1", "--config",
                          os.path.join(ROOT, "configs", "size_s.toml")], capture_output=True,
                         text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "det_evals/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["NR"] == 101 and d["ms_per_step"] > 0
    import bench
    assert d["metric"] == bench.METRIC
