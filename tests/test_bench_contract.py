"""bench.py's JSON contract, checked on the host: the reference arm (the
reference's own CPU path on the host cores) prints one line with the keys
the driver reads, and the profiling-only workloads refuse to run as a
benchmark."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*argv, timeout=600):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *argv], cwd=ROOT, capture_output=True,
                          text=True, timeout=timeout)


def test_reference_arm_line():
    r = _bench("--impl", "reference", "--steps", "1", "--warmup", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 1
    assert d["value"] > 0 and d["higher_is_better"] is True and d["unit"] == "Mpix/s"
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


def test_neighbourhood_workloads_need_a_gpu():
    """erode / median3 / median5 time per-image calls on a GPU; without one
    they exit 2 with a message instead of a traceback."""
    for w in ("erode", "median3", "median5"):
        r = _bench("--workload", w, timeout=120)
        assert r.returncode == 2 and "needs a GPU" in r.stderr, (w, r.stderr[-500:])
