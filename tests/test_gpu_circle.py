"""Canonic-coset circle FFT and circle LDE over M31 on the GPU, bit for bit
against the oracle (oracle/oracle.c orc_circle_*), which tests/test_oracle.py
pins to a direct evaluation of the circle-polynomial basis (so the LDE is
checked to be a genuine low-degree extension).  No Stwo vectors exist here
(the reference comments Stwo out, tests/ntt_cross_validation.rs:281-298), so
agreement with Stwo itself is not pinned."""
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


@pytest.mark.parametrize("log_n,batch", [(1, 2), (4, 3), (8, 64), (12, 2), (13, 1), (16, 3), (20, 2), (9, 777)])
def test_circle_ntt_matches_oracle(ctx, log_n, batch):
    c = sfntt.CircleLde(ctx)
    x = O.lcg(batch << log_n, 10 + log_n, MP)
    ev, _ = c.ntt(x, log_n, batch)
    assert np.array_equal(ev, O.circle_ntt(x, log_n, batch))
    back, _ = c.ntt(ev, log_n, batch, inverse=True)
    assert np.array_equal(back, x)


@pytest.mark.parametrize("log_n,batch,added", [(0, 3, 1), (1, 2, 2), (5, 3, 3), (8, 4, 1), (12, 3, 1), (13, 2, 1),
                                                (14, 2, 2), (16, 3, 1), (17, 1, 3), (15, 3, 4), (20, 2, 1)])
def test_circle_lde_matches_oracle(ctx, log_n, batch, added):
    x = O.lcg(batch << log_n, 30 + log_n, MP)
    r = sfntt.CircleLde(ctx).execute(x, log_n, batch, added)
    assert np.array_equal(r.data, O.circle_lde(x, log_n, batch, added, threads=8))


def test_circle_lde_full_size_low_degree(ctx):
    """2^20 x 64, 2x: sampled columns against the oracle; interpolating the
    extension on the bigger coset gives the input's coefficients then zeros."""
    import torch
    log_n, batch, added = 20, 64, 1
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    x = O.lcg(batch << log_n, 2027, MP)
    c = sfntt.CircleLde(ctx)
    c.prepare(log_n, added)
    d_in = torch.from_numpy(x.view(np.int32).copy()).cuda()
    d_out = torch.empty(batch * n_ext, dtype=torch.int32, device="cuda")
    c.execute_dev(d_in.data_ptr(), d_out.data_ptr(), log_n, batch, added)
    c.ntt_dev(d_in.data_ptr(), log_n, batch, inverse=True)     # coefficients of the input
    c.ntt_dev(d_out.data_ptr(), log_n + added, batch, inverse=True)
    torch.cuda.synchronize()
    coeffs = d_in.cpu().numpy().view(np.uint32).reshape(batch, n)
    ext = d_out.cpu().numpy().view(np.uint32).reshape(batch, n_ext)
    assert np.array_equal(ext[:, :n], coeffs)
    assert not ext[:, n:].any()
    r = c.execute(x, log_n, batch, added)
    for col in (0, batch // 2, batch - 1):
        assert np.array_equal(r.data[col * n_ext:(col + 1) * n_ext], O.circle_lde(x[col * n:(col + 1) * n], log_n, 1, added))
