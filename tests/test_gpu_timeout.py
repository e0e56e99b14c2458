"""Failure detection without a GPU fault: the tile engine's bounded mbarrier
wait, run on a barrier that nothing arrives on, gives up after its limit,
raises the context's error flag (SFNTT_TIMEOUT) and leaves the context usable."""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SFNTT_TIMEOUT = 8


def test_wait_that_runs_out_reports_timeout_and_context_survives():
    ctx = sfntt.Context(0)
    assert ctx.selftest_bounded_wait(2_000_000, arrive=False) == SFNTT_TIMEOUT  # 2 ms, nothing arrives
    assert ctx.selftest_bounded_wait(2_000_000, arrive=True) == 0  # the arrival completes the phase
    assert ctx.selftest_bounded_wait(50_000, arrive=False) == SFNTT_TIMEOUT
    # the flag was consumed; the same context still computes exactly
    x = O.lcg(1 << 14, 3, O.BB_P, monty=True)
    y = x.copy()
    sfntt.BbCudaCtGsR4(ctx).forward_ntt(y)
    assert np.array_equal(y, O.bb_forward(x))
    sfntt.BbCudaCtGsR4(ctx).inverse_ntt(y)
    assert np.array_equal(y, x)
    r = sfntt.CosetLdeBatch(ctx).execute(O.lcg(2 << 13, 4, O.BB_P, monty=True), 13, 2, 1)
    assert r.data.size == 2 << 14
