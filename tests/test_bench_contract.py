"""bench.py's command line and the reference arm's JSON line (the reference
CPU path timed on the host: runs without a GPU, here on a tiny shape)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _bench(*args: str, timeout: int = 300) -> subprocess.CompletedProcess:
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True,
                          timeout=timeout, cwd=ROOT)


def test_help_lists_the_workloads():
    r = _bench("--help")
    assert r.returncode == 0, r.stderr
    for w in ("lde", "uneven", "served", "table", "ntt", "layout"):
        assert w in r.stdout, w


def test_reference_arm_prints_one_contract_line():
    r = _bench("--impl", "reference", "--log-n", "10", "--batch", "4", "--steps", "1", "--warmup", "1")
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, lines
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "ms" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"]
    assert "workload" in d["config"] and d["config"]["parallelism"] == "single GPU"
    assert d["step_stats"]["n"] == 1


@pytest.mark.gpu
def test_gpu_arm_prints_one_contract_line():
    r = _bench("--log-n", "14", "--batch", "16", "--steps", "3", "--warmup", "3", "--no-secondary", "--no-served",
               "--no-uneven", "--cpu-seconds", "1", "--e2e-steps", "2", timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, lines
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e",
              "gpu_launches", "clocks"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    assert d["gpu_launches"] > 0
    assert {"bound", "achieved", "peak", "unit", "frac", "traffic"} <= set(d["roofline"])
    assert {"value", "unit", "cores", "kind", "sample"} <= set(d["cpu_baseline"])
    assert d["e2e"]["h2d_bytes_per_step"] == 16 << 16 and d["e2e"]["d2h_bytes_per_step"] == 2 * (16 << 16)
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(d["clocks"])
    st = d["step_stats"]
    assert st["n"] == 3 and st["min_ms"] <= st["median_ms"] <= st["max_ms"] and st["cv_pct"] >= 0
