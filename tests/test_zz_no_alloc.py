"""The allocation-free NTT entry point (sfntt_stockham_noalloc).

It exists for callers that cannot allocate device memory while they run a
transform -- a prover with a memory pool sized once at start-up, an embedder
that accounts for every device byte, a process that forbids allocation after
initialisation.  Its ping-pong scratch is a fixed file-scope device array, so
this test checks, through the C ABI, that it returns exactly what the regular
Stockham path (variant V3, which allocates its scratch lazily) returns, twice
in a row (the array keeps the previous call's contents), for both fields and
both directions, and that sizes beyond the array are rejected.  The file is
named to be collected last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import sfntt
from sfntt import _ffi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_WORDS = 1 << 20


def _dev(arr):
    import torch
    return torch.from_numpy(arr.view(np.int32).copy()).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.fixture(scope="module")
def ctx():
    return sfntt.Context(0)


@pytest.mark.parametrize("field", [sfntt.FIELD_BABYBEAR, sfntt.FIELD_M31])
@pytest.mark.parametrize("inverse", [0, 1])
@pytest.mark.parametrize("log_n,batch", [(10, 3), (13, 4), (16, 16), (20, 1)])
def test_noalloc_matches_stockham_twice(ctx, field, inverse, log_n, batch):
    import torch
    L = _ffi.lib()
    p = O.BB_P if field == sfntt.FIELD_BABYBEAR else O.M31_P
    ctx.prepare(field, log_n)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        x = O.lcg(batch << log_n, 1000 * call + log_n + 7 * inverse, p, monty=(field == sfntt.FIELD_BABYBEAR))
        ref = _dev(x)
        fn = L.sfntt_inverse_dev if inverse else L.sfntt_forward_dev
        assert fn(ctx.handle, field, sfntt.V3, ref.data_ptr(), log_n, batch, stream) == 0
        got = _dev(x)
        st = L.sfntt_stockham_noalloc(ctx.handle, field, inverse, got.data_ptr(), log_n, batch, stream)
        assert st == 0, L.sfntt_last_error(ctx.handle)
        torch.cuda.synchronize()
        assert np.array_equal(_host(got), _host(ref)), (call, field, inverse, log_n, batch)


def test_noalloc_rejects_oversize_and_cold_tables(ctx):
    import torch
    L = _ffi.lib()
    big = torch.zeros(2 * MAX_WORDS, dtype=torch.int32, device="cuda")
    ctx.prepare(sfntt.FIELD_BABYBEAR, 20)
    assert L.sfntt_stockham_noalloc(ctx.handle, sfntt.FIELD_BABYBEAR, 0, big.data_ptr(), 20, 2, None) == 1
    assert b"exceeds" in L.sfntt_last_error(ctx.handle)
    fresh = sfntt.Context(0)
    st = L.sfntt_stockham_noalloc(fresh.handle, sfntt.FIELD_M31, 0, big.data_ptr(), 12, 1, None)
    assert st == 9 and b"sfntt_prepare" in L.sfntt_last_error(fresh.handle)
    fresh.close()
