"""CM31 = M31[i]/(i^2+1) on the GPU against the oracle, bit for bit.

The reference plans the M31 quadratic extension (TODOS.md:27-31) without code;
the oracle's CM31 functions (pinned in tests/test_oracle.py: the complex
product, i^2 = -1, the transform as the M31 transform of each coordinate,
C-linearity) are the checker.
"""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from oracle import oracle as O

pytestmark = pytest.mark.gpu
MP = O.M31_P


@pytest.fixture(scope="module")
def ctx():
    return sfntt.default_context(0)


def pairs(n_pairs, seed):
    return O.lcg(2 * n_pairs, seed, MP)


@pytest.mark.parametrize("log_n,batch", [(1, 3), (5, 2), (10, 1), (12, 4), (13, 3), (16, 2), (20, 2), (8, 2048)])
def test_cm31_ntt_matches_oracle(ctx, log_n, batch):
    x = pairs(batch << log_n, 100 + log_n)
    e = sfntt.Cm31Ntt(ctx)
    fw, _ = e.forward_batch_gpu(x, log_n, batch)
    assert np.array_equal(fw, O.cm31_ntt(x, log_n, batch))
    back, _ = e.inverse_batch_gpu(fw, log_n, batch)
    assert np.array_equal(back, x)


def test_cm31_device_calls_and_product(ctx):
    import torch
    log_n, batch = 14, 3
    n = batch << log_n
    a, b = pairs(n, 1), pairs(n, 2)
    e = sfntt.Cm31Ntt(ctx)
    e.prepare(log_n, batch)
    da = torch.from_numpy(a.view(np.int32).copy()).cuda()
    db = torch.from_numpy(b.view(np.int32).copy()).cuda()
    dc = torch.empty_like(da)
    e.mul_dev(da.data_ptr(), db.data_ptr(), dc.data_ptr(), n)
    e.forward_dev(da.data_ptr(), log_n, batch)
    torch.cuda.synchronize()
    assert np.array_equal(dc.cpu().numpy().view(np.uint32), O.cm31_mul(a, b))
    assert np.array_equal(da.cpu().numpy().view(np.uint32), O.cm31_ntt(a, log_n, batch))
    e.inverse_dev(da.data_ptr(), log_n, batch)
    torch.cuda.synchronize()
    assert np.array_equal(da.cpu().numpy().view(np.uint32), a)


def test_cm31_rejects_bad_sizes(ctx):
    e = sfntt.Cm31Ntt(ctx)
    with pytest.raises(sfntt.InvalidSize):
        e.forward_batch_gpu(np.zeros(100, np.uint32), 4, 3)
    with pytest.raises(sfntt.InvalidSize):
        e.forward_batch_gpu(np.zeros(2 << 31 >> 31, np.uint32), 31, 1)
