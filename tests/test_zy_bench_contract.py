"""bench.py's JSON line: the keys and types its readers rely on, for the reference arm (the
CPU restatement timed on the host, here on the CPU) and this build's arm (on a GPU)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, timeout):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                         timeout=timeout, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def _common(line):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "e2e"):
        assert k in line, k
    assert line["metric"] == "TGV DOF-updates/s/stage" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["config"]["workload"] == "tgv_viscous_24_p5"
    assert set(line["e2e"]) >= {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"}


def test_reference_arm_line():
    line = _run(["--impl", "reference", "--steps", "1", "--warmup", "1"], timeout=600)
    _common(line)
    assert line["impl"] == "reference"
    assert line["cpu_baseline"]["kind"] in ("port", "reference") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]


@pytest.mark.gpu
def test_gpu_arm_line():
    line = _run(["--steps", "3", "--warmup", "3", "--no-cpu-baseline"], timeout=900)
    _common(line)
    assert line["n_gpus"] == 1 and line["steps"] == 3 and line["warmup"] == 3
    assert line["gpu_launches"] > 0
    r = line["roofline"]
    # the stage kernel's binding roof is its FP64 pipe (TFLOP/s against a measured DGEMM); the
    # HBM figures ride along under "hbm"
    assert (r["bound"], r["unit"]) in (("hbm", "GB/s"), ("tensor", "TFLOP/s"), ("fp64", "TFLOP/s"), ("fp32", "TFLOP/s"))
    assert r["hbm"]["unit"] == "GB/s" and r["hbm"]["achieved"] > 0
    assert r["achieved"] > 0 and r["peak"] > 0 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert r["traffic"] is None or isinstance(r["traffic"], float)
    assert line["e2e"]["h2d_bytes_per_step"] > 0 and line["e2e"]["d2h_bytes_per_step"] > 0
    c = line["clocks"]
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(c)
