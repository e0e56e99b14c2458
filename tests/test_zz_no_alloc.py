"""The allocation-free NTT entry point (sfntt_stockham_noalloc).

It exists for callers that cannot allocate device memory while they run a
transform -- a prover with a memory pool sized once at start-up, an embedder
that accounts for every device byte, a process that forbids allocation after
initialisation.  Its ping-pong scratch is a fixed file-scope device array.
Through the C ABI this test checks, for all three fields and both
directions, twice in a row (the array keeps the previous call's contents):

* that every column equals the oracle (the reference's CPU NTT restated) and
  the regular Stockham path (variant V3, which allocates its scratch lazily);
* that the calls after the first on a device change the device's free memory
  by nothing (the first call resolves the array's address, which under lazy
  module loading may load the module);
* that sizes beyond the array, and twiddles that are not resident, are
  rejected.

The file is named to be collected last.
"""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from sfntt import _ffi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_WORDS = 1 << 20
BB, KB, M31 = sfntt.FIELD_BABYBEAR, sfntt.FIELD_KOALABEAR, sfntt.FIELD_M31
P = {BB: O.BB_P, KB: O.KB_P, M31: O.M31_P}


def _dev(arr):
    import torch
    return torch.from_numpy(arr.view(np.int32).copy()).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def _oracle(field, inverse, x, log_n, batch):
    if field == BB:
        return (O.bb_inverse_batch if inverse else O.bb_forward_batch)(x, log_n, batch, threads=8)
    if field == KB:
        return (O.kb_inverse_batch if inverse else O.kb_forward_batch)(x, log_n, batch, threads=8)
    n = 1 << log_n
    fn = O.m31_inverse if inverse else O.m31_forward
    return np.concatenate([fn(x[c * n:(c + 1) * n]) for c in range(batch)])


@pytest.fixture(scope="module")
def ctx():
    return sfntt.Context(0)


@pytest.mark.parametrize("field", [BB, KB, M31], ids=["bb", "kb", "m31"])
@pytest.mark.parametrize("inverse", [0, 1])
@pytest.mark.parametrize("log_n,batch", [(10, 3), (13, 4), (16, 16), (20, 1)])
def test_noalloc_matches_oracle_twice(ctx, field, inverse, log_n, batch):
    import torch
    L = _ffi.lib()
    ctx.prepare(field, log_n)
    stream = torch.cuda.current_stream().cuda_stream
    # the first call on a device resolves the scratch address (set-up)
    warm = torch.zeros(batch << log_n, dtype=torch.int32, device="cuda")
    assert L.sfntt_stockham_noalloc(ctx.handle, field, inverse, warm.data_ptr(), log_n, batch, stream) == 0
    torch.cuda.synchronize()
    for call in range(2):
        x = O.lcg(batch << log_n, 1000 * call + log_n + 7 * inverse, P[field], monty=(field != M31))
        ref = _dev(x)
        fn = L.sfntt_inverse_dev if inverse else L.sfntt_forward_dev
        assert fn(ctx.handle, field, sfntt.V3, ref.data_ptr(), log_n, batch, stream) == 0
        got = _dev(x)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        st = L.sfntt_stockham_noalloc(ctx.handle, field, inverse, got.data_ptr(), log_n, batch, stream)
        assert st == 0, L.sfntt_last_error(ctx.handle)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, ("device memory changed across the call", free0 - free1)
        out = _host(got)
        assert np.array_equal(out, _oracle(field, inverse, x, log_n, batch)), (call, field, inverse, log_n, batch)
        assert np.array_equal(out, _host(ref)), (call, field, inverse, log_n, batch)


def test_noalloc_rejects_oversize_and_cold_tables(ctx):
    import torch
    L = _ffi.lib()
    big = torch.zeros(2 * MAX_WORDS, dtype=torch.int32, device="cuda")
    ctx.prepare(BB, 20)
    assert L.sfntt_stockham_noalloc(ctx.handle, BB, 0, big.data_ptr(), 20, 2, None) == 1
    assert b"exceeds" in L.sfntt_last_error(ctx.handle)
    fresh = sfntt.Context(0)
    st = L.sfntt_stockham_noalloc(fresh.handle, M31, 0, big.data_ptr(), 12, 1, None)
    assert st == 9 and b"sfntt_prepare" in L.sfntt_last_error(fresh.handle)
    fresh.close()
