"""KoalaBear (p = 2^31 - 2^24 + 1) on the GPU against the oracle, bit for bit.

The reference lists KoalaBear as planned (README.md:20) and has no code for
it, so the oracle's KoalaBear functions (the BabyBear restatement over
KoalaBear's constants, pinned in tests/test_oracle.py against a direct DFT and
coset evaluation) are the checker.  The cases follow the BabyBear parity tests:
every algorithm variant, batches, many small columns, the fused and unfused
coset LDE on both tile engines, the natural-order convention, uneven batches
in a CUDA graph, and on-device Montgomery conversion.
"""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KB = sfntt.FIELD_KOALABEAR
KB_BACKENDS = [sfntt.KbCudaCtDitR2, sfntt.KbBatchNtt, sfntt.KbCudaStockhamR2, sfntt.KbCudaCtGsR4]


@pytest.fixture(scope="module")
def ctx():
    return sfntt.default_context(0)


def kdata(n, seed):
    return O.lcg(n, seed, O.KB_P, monty=True)


@pytest.mark.parametrize("cls", KB_BACKENDS)
@pytest.mark.parametrize("log_n", [1, 2, 5, 10, 12, 13, 16, 18, 20])
def test_kb_forward_inverse(ctx, cls, log_n):
    b = cls(ctx)
    x = kdata(1 << log_n, 500 + log_n)
    fw, _ = b.forward_ntt_gpu(x, log_n)
    assert np.array_equal(fw, O.kb_forward(x))
    if cls is sfntt.KbCudaCtDitR2:
        with pytest.raises(sfntt.Unsupported):
            b.inverse_ntt_gpu(fw, log_n)
        return
    back, _ = b.inverse_ntt_gpu(fw, log_n)
    assert np.array_equal(back, x)


def test_kb_largest_size_and_limits(ctx):
    b = sfntt.KbCudaCtGsR4(ctx)
    log_n = 24  # two-adicity of KoalaBear
    x = kdata(1 << log_n, 24)
    fw, _ = b.forward_ntt_gpu(x, log_n)
    assert np.array_equal(fw, O.kb_forward(x))
    back, _ = b.inverse_ntt_gpu(fw, log_n)
    assert np.array_equal(back, x)
    with pytest.raises(sfntt.InvalidSize):
        b.forward_ntt_gpu(np.zeros(1 << 25, np.uint32), 25)


@pytest.mark.parametrize("log_n,batch", [(1, 5), (8, 64), (10, 7), (12, 2), (14, 16), (20, 3)])
def test_kb_batch_equals_single(ctx, log_n, batch):
    b = sfntt.KbBatchNtt(ctx)
    x = kdata(batch << log_n, 600 + log_n)
    fw, _ = b.forward_ntt_batch_gpu(x, log_n, batch)
    assert np.array_equal(fw, O.kb_forward_batch(x, log_n, batch, threads=8))
    back, _ = b.inverse_ntt_batch_gpu(fw, log_n, batch)
    assert np.array_equal(back, x)


@pytest.mark.parametrize("log_n,batch", [(8, 4096), (10, 1024), (9, 777)])
def test_kb_many_small_columns(ctx, log_n, batch):
    b = sfntt.KbBatchNtt(ctx)
    x = kdata(batch << log_n, 700 + log_n)
    fw, _ = b.forward_ntt_batch_gpu(x, log_n, batch)
    assert np.array_equal(fw, O.kb_forward_batch(x, log_n, batch, threads=8))
    back, _ = b.inverse_ntt_batch_gpu(fw, log_n, batch)
    assert np.array_equal(back, x)


def test_kb_pointwise_product(ctx):
    """Polynomial product through the transform (ntt_cross_validation.rs:113-148 over KoalaBear)."""
    b = sfntt.KbCudaCtGsR4(ctx)
    to = [O.kb_to_monty(v) for v in (1, 2, 0, 0)], [O.kb_to_monty(v) for v in (3, 4, 0, 0)]
    fa, _ = b.forward_ntt_gpu(np.array(to[0], np.uint32), 2)
    fb, _ = b.forward_ntt_gpu(np.array(to[1], np.uint32), 2)
    prod = np.empty(4, np.uint32)
    b.pointwise_mul(fa, fb, prod)
    c, _ = b.inverse_ntt_gpu(prod, 2)
    assert [O.kb_from_monty(int(v)) for v in c] == [3, 10, 8, 0]


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("log_n,batch,added", [(8, 4, 1), (0, 3, 1), (5, 3, 3), (12, 8, 1), (11, 5, 4), (6, 2, 5),
                                                (13, 2, 1), (14, 3, 2), (16, 4, 1), (18, 2, 1),
                                                (13, 16, 1), (15, 17, 1), (16, 33, 3)])
def test_kb_coset_lde_matches_oracle(ctx, fused, log_n, batch, added):
    x = kdata(batch << log_n, 800 + log_n)
    r = sfntt.KbCosetLdeBatch(ctx, fused=fused).execute(x, log_n, batch, added)
    assert np.array_equal(r.data, O.kb_coset_lde(x, log_n, batch, added, threads=8))


def test_kb_coset_lde_generator_shift_and_natural(ctx):
    """Coset g = 3 (KoalaBear's multiplicative generator) and natural-order rows."""
    sh = O.kb_to_monty(3)
    log_n, batch, added = 14, 4, 1
    x = kdata(batch << log_n, 31)
    r = sfntt.KbCosetLdeBatch(ctx).execute(x, log_n, batch, added, shift_monty=sh)
    assert np.array_equal(r.data, O.kb_coset_lde(x, log_n, batch, added, sh, threads=4))
    # natural: input rows natural, output rows natural (bit-reverse each column on both sides)
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    rev = lambda bits: np.array([int(format(k, f"0{bits}b")[::-1], 2) for k in range(1 << bits)])
    x_nat = x.reshape(batch, n)[:, rev(log_n)].ravel()
    nat = sfntt.KbCosetLdeBatch(ctx, natural=True).execute(x_nat, log_n, batch, added, shift_monty=sh).data
    assert np.array_equal(nat.reshape(batch, n_ext), r.data.reshape(batch, n_ext)[:, rev(log_n + added)])


def test_kb_natural_lde_full_size_sampled_columns(ctx):
    """2^20 x 8 natural-order rows (the mirrored network, strided passes with
    chunk-staged twiddles): sampled columns against the oracle."""
    log_n, batch, added = 20, 8, 1
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    rev = lambda bits: np.array([int(format(k, f"0{bits}b")[::-1], 2) for k in range(1 << bits)])
    r_n, r_ext = rev(log_n), rev(log_n + added)
    x_nat = kdata(batch << log_n, 2027)
    got = sfntt.KbCosetLdeBatch(ctx, natural=True).execute(x_nat, log_n, batch, added).data.reshape(batch, n_ext)
    for c in (0, 3, batch - 1):
        ref = O.kb_coset_lde(x_nat[c * n:(c + 1) * n][r_n], log_n, 1, added)
        assert np.array_equal(got[c], ref[r_ext]), c


def test_kb_coset_lde_full_size_sampled_columns(ctx):
    """2^20 x 64, 2x: sampled columns against the oracle; the extension
    interpolates to a polynomial of degree < n on every column."""
    log_n, batch, added = 20, 64, 1
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    x = kdata(batch << log_n, 2026)
    r = sfntt.KbCosetLdeBatch(ctx).execute(x, log_n, batch, added)
    for c in (0, 1, batch // 2, batch - 1):
        assert np.array_equal(r.data[c * n_ext:(c + 1) * n_ext], O.kb_coset_lde(x[c * n:(c + 1) * n], log_n, 1, added)), c
    coeffs, _ = sfntt.KbBatchNtt(ctx).inverse_ntt_batch_gpu(r.data, log_n + added, batch)
    assert not coeffs.reshape(batch, n_ext)[:, n:].any()


def test_kb_lde_limits(ctx):
    lde = sfntt.KbCosetLdeBatch(ctx)
    with pytest.raises(sfntt.InvalidSize):
        lde.execute(np.zeros(100, np.uint32), 8, 4, 1)
    with pytest.raises(sfntt.InvalidSize):  # log_n + added_bits + 1 > 24
        lde.execute(np.zeros(1 << 20, np.uint32), 20, 1, 4)


@pytest.mark.parametrize("plan", [sfntt.PLAN_TMA, sfntt.PLAN_TMA_FOUR_STEP, sfntt.PLAN_TILE])
def test_kb_items_in_uneven_graph(ctx, plan):
    import torch
    shapes = [(14, 3, 2), (16, 2, 1), (9, 5, 1), (13, 16, 1)]
    items, bufs = [], []
    for k, (ln, b, ab) in enumerate(shapes):
        x = kdata(b << ln, 40 + k)
        d_in = torch.from_numpy(x.view(np.int32).copy()).cuda()
        d_out = torch.zeros(b << (ln + ab), dtype=torch.int32, device="cuda")
        items.append({"field": KB, "log_n": ln, "batch": b, "added_bits": ab, "plan": plan,
                      "d_in": d_in.data_ptr(), "d_out": d_out.data_ptr()})
        bufs.append((x, d_in, d_out))
    batch = sfntt.LdeBatch(ctx, items)
    batch.prepare()
    g = batch.graph(lanes=4)
    g.launch()
    torch.cuda.synchronize()
    for (ln, b, ab), (x, _, d_out) in zip(shapes, bufs):
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), O.kb_coset_lde(x, ln, b, ab, threads=8))
    g.close()


def test_kb_monty_conversion_on_device(ctx):
    import torch
    v = O.lcg(100_003, 5, O.KB_P)
    d = torch.from_numpy(v.view(np.int32).copy()).cuda()
    sfntt.convert_monty_dev(ctx, KB, d.data_ptr(), v.size, to_monty=True)
    torch.cuda.synchronize()
    m = d.cpu().numpy().view(np.uint32)
    assert np.array_equal(m[:1000], np.array([O.kb_to_monty(int(a)) for a in v[:1000]], np.uint32))
    sfntt.convert_monty_dev(ctx, KB, d.data_ptr(), v.size, to_monty=False)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), v)
    with pytest.raises(sfntt.InvalidArgument):
        sfntt.convert_monty_dev(ctx, sfntt.FIELD_M31, d.data_ptr(), v.size, to_monty=True)
