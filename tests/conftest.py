"""Shared pytest setup: markers, import paths, fixture loading."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "small-field-metal-ntt_b200"
for p in (ROOT, PKG):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


@pytest.fixture(scope="session")
def golden():
    meta = json.loads((ROOT / "tests" / "golden" / "golden.json").read_text())
    arrays = dict(np.load(ROOT / "tests" / "golden" / "golden.npz"))
    return meta, arrays
