"""Synthetic workload generators (host logic, no GPU): the uneven batch and
the served stream draw what their configurations state, deterministically."""
from __future__ import annotations

import numpy as np

import sfntt


def test_uneven_workload_ranges_and_seed():
    a = sfntt.uneven_workload(64, seed=2024)
    assert a == sfntt.uneven_workload(64, seed=2024)
    assert {it["field"] for it in a} == {sfntt.FIELD_M31, sfntt.FIELD_BABYBEAR}
    assert all(12 <= it["log_n"] <= 22 and 1 <= it["batch"] <= 128 for it in a)
    assert {it["added_bits"] for it in a} <= {0, 1, 2}


def test_served_workload_shape():
    reqs, arr = sfntt.served_workload(4000, rate=500.0, seed=2025)
    assert len(reqs) == len(arr) == 4000
    assert np.all(np.diff(arr) >= 0) and arr[0] > 0
    # Poisson arrivals: mean inter-arrival 1 / rate
    assert abs(np.diff(arr).mean() - 1 / 500.0) < 0.1 / 500.0
    logs = np.array([it["log_n"] for it in reqs])
    assert logs.min() >= 14 and logs.max() <= 22
    share_18_20 = np.mean((logs >= 18) & (logs <= 20))
    assert share_18_20 > 0.55  # weighted toward 18..20
    cols = np.array([it["batch"] for it in reqs])
    assert cols.min() >= 8 and cols.max() <= 256
    assert {it["added_bits"] for it in reqs} == {1, 2}
    fields = np.array([it["field"] for it in reqs])
    assert 0.45 < fields.mean() < 0.55
    # the same trace at another rate: same requests, arrivals scaled
    reqs2, arr2 = sfntt.served_workload(4000, rate=50.0, seed=2025)
    assert reqs2 == reqs and np.allclose(arr2 * 50.0, arr * 500.0)
