"""Output conventions: natural row order (Plonky3's coset_lde_batch) and the
row-major Merkle-commitment layout (sfntt_layout*, SFNTT_LDE_NATURAL).

The expected values are numpy permutations of the oracle's outputs (the
reference's bit-reversed convention)."""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bitrev_idx(log_n: int) -> np.ndarray:
    n = 1 << log_n
    r = np.zeros(n, dtype=np.int64)
    for b in range(log_n):
        r |= ((np.arange(n) >> b) & 1) << (log_n - 1 - b)
    return r


def _natural(x: np.ndarray, log_n: int, batch: int) -> np.ndarray:
    return x.reshape(batch, 1 << log_n)[:, _bitrev_idx(log_n)].reshape(-1)


@pytest.fixture(scope="module")
def ctx():
    return sfntt.Context(0)


@pytest.mark.parametrize("log_n,batch", [(0, 3), (1, 1), (3, 5), (5, 33), (9, 2), (10, 1), (11, 7), (12, 64),
                                         (14, 3), (16, 1),
                                         # wide tiles: partial column blocks, one row block, tile pairs
                                         (6, 100), (13, 65), (15, 130), (17, 3), (5, 128), (9, 300)])
def test_layout_matches_numpy(ctx, log_n, batch):
    n = 1 << log_n
    x = O.lcg(batch * n, 91 + log_n + batch, O.M31_P)
    soa = x.reshape(batch, n)
    nat, _ = sfntt.layout(x, log_n, batch, sfntt.LAYOUT_NATURAL, ctx)
    assert np.array_equal(nat, _natural(x, log_n, batch))
    rows, _ = sfntt.layout(x, log_n, batch, sfntt.LAYOUT_ROW_MAJOR, ctx)
    assert np.array_equal(rows, soa.T.reshape(-1))
    both, _ = sfntt.layout(x, log_n, batch, sfntt.LAYOUT_NATURAL | sfntt.LAYOUT_ROW_MAJOR, ctx)
    assert np.array_equal(both, soa[:, _bitrev_idx(log_n)].T.reshape(-1))
    same, _ = sfntt.layout(x, log_n, batch, 0, ctx)
    assert np.array_equal(same, x)


@pytest.mark.parametrize("log_n,batch", [(4, 3), (10, 2), (13, 5), (20, 4)])
def test_natural_in_place_is_an_involution(ctx, log_n, batch):
    import torch
    x = O.lcg(batch << log_n, 5 + log_n, O.BB_P)
    d = torch.from_numpy(x.view(np.int32).copy()).cuda()
    sfntt.layout_dev(ctx, d.data_ptr(), d.data_ptr(), log_n, batch, sfntt.LAYOUT_NATURAL)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), _natural(x, log_n, batch))
    sfntt.layout_dev(ctx, d.data_ptr(), d.data_ptr(), log_n, batch, sfntt.LAYOUT_NATURAL)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), x)


def test_layout_rejects_bad_buffers(ctx):
    import torch
    d = torch.zeros(1 << 12, dtype=torch.int32, device="cuda")
    with pytest.raises(sfntt.InvalidArgument):  # row-major is out of place
        sfntt.layout_dev(ctx, d.data_ptr(), d.data_ptr(), 10, 4, sfntt.LAYOUT_ROW_MAJOR)
    with pytest.raises(sfntt.InvalidArgument):  # overlapping, not identical
        sfntt.layout_dev(ctx, d.data_ptr(), d.data_ptr() + 64, 10, 2, sfntt.LAYOUT_NATURAL)
    with pytest.raises(sfntt.InvalidArgument):
        sfntt.layout_dev(ctx, d.data_ptr(), d.data_ptr() + 8192, 10, 1, 4)
    with pytest.raises(sfntt.InvalidSize):
        sfntt.layout(np.zeros(10, dtype=np.uint32), 2, 3, sfntt.LAYOUT_NATURAL, ctx)


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("log_n,batch,added,shift", [(10, 3, 1, 0), (13, 2, 2, 0), (14, 3, 1, 31), (6, 2, 3, 31),
                                                     (0, 2, 2, 0), (16, 2, 1, 31),
                                                     # 2x, 2^13..2^20: the mirrored network without bit reversals
                                                     (13, 1, 1, 0), (13, 3, 1, 31), (15, 5, 1, 0), (17, 16, 1, 31),
                                                     (18, 2, 1, 7), (12, 4, 1, 31)])
def test_natural_lde_is_plonky3_convention(ctx, fused, log_n, batch, added, shift):
    """Natural-order evaluations in, natural-order rows out: the reference LDE
    conjugated by the bit-reversal permutation on both sides."""
    shift_monty = O.bb_to_monty(shift) if shift else 0
    x_nat = O.lcg(batch << log_n, 300 + log_n, O.BB_P, monty=True)
    x_br = _natural(x_nat, log_n, batch)  # bit reversal is an involution
    ref = O.bb_coset_lde(x_br, log_n, batch, added, shift_monty=shift_monty, threads=4)
    expect = _natural(ref, log_n + added, batch)
    got = sfntt.CosetLdeBatch(ctx, fused=fused, natural=True).execute(x_nat, log_n, batch, added, shift_monty).data
    assert np.array_equal(got, expect)


def test_natural_lde_device_path_2_20(ctx):
    """The full-width device path (TMA passes) with natural order: sampled
    columns against the oracle."""
    import torch
    log_n, batch, added = 20, 8, 1
    x_nat = O.lcg(batch << log_n, 4242, O.BB_P, monty=True)
    d_in = torch.from_numpy(x_nat.view(np.int32).copy()).cuda()
    d_out = torch.empty(batch << (log_n + added), dtype=torch.int32, device="cuda")
    sfntt.CosetLdeBatch(ctx, natural=True).execute_dev(d_in.data_ptr(), d_out.data_ptr(), log_n, batch, added)
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().view(np.uint32).reshape(batch, -1)
    for c in (0, 5):
        col = x_nat.reshape(batch, -1)[c]
        ref = O.bb_coset_lde(_natural(col, log_n, 1), log_n, 1, added, threads=8)
        assert np.array_equal(got[c], _natural(ref, log_n + added, 1)), c


def test_natural_lde_in_graph_with_and_without_scratch(ctx):
    """Captured in a CUDA graph the natural-order 2x LDE either takes the
    no-bit-reversal route (scratch already reserved by an earlier call) or
    falls back to the bit-reversal route (fresh context): same results."""
    import torch
    log_n, batch, added = 14, 4, 1
    x_nat = O.lcg(batch << log_n, 77, O.BB_P, monty=True)
    ref = _natural(O.bb_coset_lde(_natural(x_nat, log_n, batch), log_n, batch, added, threads=4), log_n + added, batch)
    for warm in (True, False):
        c = sfntt.Context(0)
        c.prepare_lde(sfntt.FIELD_BABYBEAR, log_n, added)
        lde = sfntt.CosetLdeBatch(c, natural=True)
        d_in = torch.from_numpy(x_nat.view(np.int32).copy()).cuda()
        d_out = torch.zeros(batch << (log_n + added), dtype=torch.int32, device="cuda")
        if warm:
            lde.execute_dev(d_in.data_ptr(), d_out.data_ptr(), log_n, batch, added)
            torch.cuda.synchronize()
            d_out.zero_()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            lde.execute_dev(d_in.data_ptr(), d_out.data_ptr(), log_n, batch, added,
                            stream=torch.cuda.current_stream().cuda_stream)
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), ref), warm
        del g
        c.close()
