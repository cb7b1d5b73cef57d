"""The JSON line of bench.py, which the benchmark driver reads: the keys and
their meaning, on small grids.

CPU: the reference arm (the oracle port on the host cores) prints one line
with impl "reference", its cpu_baseline and an e2e of its own value.  GPU:
the default arm prints the metric, the whole-job value, the timing
protocol, clocks, the roofline of the dominant kernel from the timed steps,
kernel-class times that add up to the step time, the launch count, the
float64 arm's speed-up and the end-to-end figure with its copied bytes.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _line(args, timeout=600):
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT,
                       env=env, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_reference_arm_line():
    d = _line(["--impl", "reference", "--n", "24", "--steps", "1", "--warmup", "0"])
    assert d["impl"] == "reference" and d["unit"] == "zone-updates/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


@pytest.mark.gpu
def test_gpu_arm_line():
    steps = 4
    d = _line(["--n", "48", "--steps", str(steps), "--warmup", "3", "--no-cpu"])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "gpu_launches", "clocks", "roofline", "e2e"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == steps and d["warmup"] == 3
    assert d["scaling"] == "weak" and d["finite"] is True
    assert abs(d["value"] - 48 ** 3 * steps / (d["ms_per_step"] * steps / 1e3)) < 1e-6 * d["value"]
    assert d["gpu_launches"] >= 20 * steps
    assert d["clocks"]["samples"] >= 1 and "reasons" in d["clocks"]
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] > 0
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3
    # kernel classes of the timed steps add up to the step time
    assert d["kernel_times_from"] == "the timed steps"
    ks = sum(d["kernel_ms_per_step"].values())
    assert abs(ks - d["ms_per_step"]) < 0.05 * d["ms_per_step"], (ks, d["ms_per_step"])
    # the float64 arm ran (its speed-up is a property of 256^3, not of 48^3,
    # where the learned con2prim's persistent grid is mostly idle)
    assert d["fp64_value"] > 0 and d["speedup_vs_fp64"] > 0
    e = d["e2e"]
    nbytes = 11 * (48 + 6) ** 3 * 8
    assert e["h2d_bytes_per_step"] == nbytes and e["d2h_bytes_per_step"] == nbytes
    assert e["value"] > 0 and e["steps"] >= 8
