"""The C++ host mirror (small-field-metal-ntt_b200/cpp/sfntt.hpp): compiled
with g++ against the C ABI and the oracle, then run as a test binary."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "test_mirror.cpp"
OUT = ROOT / "tests" / "cpp" / "_build" / "test_mirror"
LIBS = [ROOT / "small-field-metal-ntt_b200" / "lib" / "libsfntt.so", ROOT / "oracle" / "liboracle.so"]


@pytest.fixture(scope="module")
def binary() -> Path:
    for lib in LIBS:
        assert lib.exists(), f"{lib} is missing: run __graft_entry__.build()"
    deps = [SRC, ROOT / "small-field-metal-ntt_b200" / "cpp" / "sfntt.hpp", ROOT / "include" / "sfntt.h", *LIBS]
    if not OUT.exists() or OUT.stat().st_mtime < max(p.stat().st_mtime for p in deps):
        OUT.parent.mkdir(parents=True, exist_ok=True)
        cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", str(SRC), "-o", str(OUT),
               f"-L{LIBS[0].parent}", "-lsfntt", f"-L{LIBS[1].parent}", "-loracle",
               "-Wl,-rpath,$ORIGIN/../../../small-field-metal-ntt_b200/lib:$ORIGIN/../../../oracle"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    return OUT


def _gpu_visible() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_mirror_host_only(binary):
    if _gpu_visible():
        pytest.skip("a GPU is visible: the parity run covers the mirror")
    r = subprocess.run([str(binary), "--no-device"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_mirror_parity(binary):
    r = subprocess.run([str(binary)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 failed" in r.stdout
