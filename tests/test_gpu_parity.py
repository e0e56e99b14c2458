"""GPU parity: every CUDA path against the C oracle, bit for bit.

Mirrors the reference's GPU test strategy (src/ntt/test_utils.rs:61-168,
tests/ntt_cross_validation.rs:186-486, src/lde/mod.rs:194-271): forward vs CPU,
round trip, edge cases (zeros, size 1, invalid / empty sizes), pointwise
product, batch == per-column, coset LDE vs coset_lde_batch_cpu.  All calls go
through the C ABI (sfntt -> libsfntt.so).
"""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from oracle import oracle as O

pytestmark = pytest.mark.gpu

BB, M31 = sfntt.FIELD_BABYBEAR, sfntt.FIELD_M31
P = {BB: O.BB_P, M31: O.M31_P}
M31_BACKENDS = [sfntt.CudaCtDitR2, sfntt.CudaCtGsR2, sfntt.CudaStockhamR2, sfntt.CudaCtGsR4]
BB_BACKENDS = [sfntt.BbCudaCtDitR2, sfntt.BbBatchNtt, sfntt.BbCudaStockhamR2, sfntt.BbCudaCtGsR4]


@pytest.fixture(scope="module")
def ctx():
    return sfntt.default_context(0)


def data(field, n, seed):
    return O.lcg(n, seed, P[field], monty=(field == BB))


def ofwd(field, x):
    return O.bb_forward(x) if field == BB else O.m31_forward(x)


def oinv(field, x):
    return O.bb_inverse(x) if field == BB else O.m31_inverse(x)


# ---- golden fixtures straight through the GPU --------------------------------
def test_gpu_matches_golden_fixtures(ctx, golden):
    meta, arr = golden
    for key, cls, inverse in (("bb_forward", sfntt.BbCudaCtGsR4, False), ("bb_inverse", sfntt.BbCudaCtGsR4, True),
                              ("m31_forward", sfntt.CudaCtGsR4, False), ("m31_inverse", sfntt.CudaCtGsR4, True)):
        b = cls(ctx)
        for case in meta[key]:
            x = arr[case["input"]].copy()
            (b.inverse_ntt if inverse else b.forward_ntt)(x)
            assert np.array_equal(x, arr[case["output"]]), (key, case["log_n"])
    lde = sfntt.CosetLdeBatch(ctx)
    for case in meta["bb_lde"]:
        if "input" not in case:
            continue
        r = lde.execute(arr[case["input"]], case["log_n"], case["batch"], case["added_bits"],
                        case.get("shift_monty", 0))
        assert np.array_equal(r.data, arr[case["output"]]), case


# ---- single-column forward / inverse, every variant ------------------------
@pytest.mark.parametrize("cls", M31_BACKENDS + BB_BACKENDS, ids=lambda c: c.NAME)
def test_forward_matches_cpu_all_sizes(ctx, cls):
    f = cls.FIELD
    b = cls(ctx)
    for log_n in range(1, 17):
        x = data(f, 1 << log_n, (1 << log_n) * 11111 + 98765)
        y = x.copy()
        b.forward_ntt(y)
        assert np.array_equal(y, ofwd(f, x)), (cls.NAME, log_n)


@pytest.mark.parametrize("cls", [c for c in M31_BACKENDS + BB_BACKENDS if c.VARIANT != sfntt.V1],
                         ids=lambda c: c.NAME)
def test_inverse_matches_cpu_and_roundtrips(ctx, cls):
    f = cls.FIELD
    b = cls(ctx)
    for log_n in range(1, 17):
        x = data(f, 1 << log_n, 7 + log_n)
        y = x.copy()
        b.inverse_ntt(y)
        assert np.array_equal(y, oinv(f, x)), (cls.NAME, log_n)
        z = x.copy()
        b.forward_ntt(z)
        assert not np.array_equal(z, x)
        b.inverse_ntt(z)
        assert np.array_equal(z, x), (cls.NAME, log_n)


@pytest.mark.parametrize("log_n", [17, 18, 20, 22, 24])
def test_bb_large_sizes_match_cpu(ctx, log_n):
    b = sfntt.BbCudaCtGsR4(ctx)
    x = data(BB, 1 << log_n, 12345 + log_n)
    fw, _ = b.forward_ntt_gpu(x, log_n)
    assert np.array_equal(fw, O.bb_forward(x))
    iv, _ = b.inverse_ntt_gpu(x, log_n)
    assert np.array_equal(iv, O.bb_inverse(x))


@pytest.mark.parametrize("log_n", [17, 18, 20])
def test_m31_large_sizes_match_cpu(ctx, log_n):
    b = sfntt.CudaCtGsR4(ctx)
    x = data(M31, 1 << log_n, 999 + log_n)
    fw, _ = b.forward_ntt_gpu(x, log_n)
    assert np.array_equal(fw, O.m31_forward(x))
    iv, _ = b.inverse_ntt_gpu(x, log_n)
    assert np.array_equal(iv, O.m31_inverse(x))


@pytest.mark.parametrize("field", [BB, M31])
def test_roundtrip_up_to_2_24(ctx, field):
    b = (sfntt.BbCudaCtGsR4 if field == BB else sfntt.CudaCtGsR4)(ctx)
    for log_n in (21, 23, 24):
        x = data(field, 1 << log_n, log_n)
        fw, _ = b.forward_ntt_gpu(x, log_n)
        back, _ = b.inverse_ntt_gpu(fw, log_n)
        assert np.array_equal(back, x), log_n
        assert np.all(fw < P[field])


def test_bb_27_bit_transform_roundtrip(ctx):
    # largest BabyBear size (two-adicity 27) goes through the three-pass plan
    log_n = 25
    b = sfntt.BbCudaCtGsR4(ctx)
    x = data(BB, 1 << log_n, 3)
    fw, _ = b.forward_ntt_gpu(x, log_n)
    back, _ = b.inverse_ntt_gpu(fw, log_n)
    assert np.array_equal(back, x)
    # linearity against a second input at the same size
    y = data(BB, 1 << log_n, 4)
    fy, _ = b.forward_ntt_gpu(y, log_n)
    s = ((x.astype(np.uint64) + y) % O.BB_P).astype(np.uint32)
    fs, _ = b.forward_ntt_gpu(s, log_n)
    assert np.array_equal(fs, ((fw.astype(np.uint64) + fy) % O.BB_P).astype(np.uint32))


# ---- edge cases (src/ntt/test_utils.rs:104-153) ------------------------------
@pytest.mark.parametrize("cls", M31_BACKENDS + BB_BACKENDS, ids=lambda c: c.NAME)
def test_edge_cases(ctx, cls):
    b = cls(ctx)
    z = np.zeros(64, np.uint32)
    b.forward_ntt(z)
    assert not z.any()
    one = np.array([O.bb_to_monty(42) if cls.FIELD == BB else 42], np.uint32)
    before = one.copy()
    b.forward_ntt(one)
    assert np.array_equal(one, before)
    for bad in (np.ones(3, np.uint32), np.zeros(0, np.uint32)):
        with pytest.raises(sfntt.InvalidSize):
            b.forward_ntt(bad)
        with pytest.raises(sfntt.InvalidSize):
            b.inverse_ntt(bad)
    if cls.VARIANT == sfntt.V1:
        with pytest.raises(sfntt.Unsupported):
            b.inverse_ntt(np.ones(8, np.uint32))
    else:
        one = before.copy()
        b.inverse_ntt(one)
        assert np.array_equal(one, before)


def test_m31_constant_poly_is_all_ones(ctx):  # ntt_cross_validation.rs:634-645
    for cls in M31_BACKENDS:
        x = np.zeros(16, np.uint32)
        x[0] = 1
        cls(ctx).forward_ntt(x)
        assert np.all(x == 1), cls.NAME


def test_m31_size_limit(ctx):
    b = sfntt.CudaCtGsR4(ctx)
    with pytest.raises(sfntt.InvalidSize):
        b.forward_ntt_gpu(np.zeros(1, np.uint32), 31)


def test_pointwise_mul(ctx):  # test_utils.rs:156-168
    m = sfntt.CudaCtGsR4(ctx)
    out = np.zeros(4, np.uint32)
    m.pointwise_mul([2, 3, 4, 5], [10, 20, 30, 40], out)
    assert list(out) == [20, 60, 120, 200]
    with pytest.raises(sfntt.InvalidSize):
        m.pointwise_mul(np.ones(4, np.uint32), np.ones(3, np.uint32), np.zeros(4, np.uint32))
    bb = sfntt.BbCudaCtGsR4(ctx)
    a, b = data(BB, 1000, 1), data(BB, 1000, 2)
    out = np.zeros(1000, np.uint32)
    bb.pointwise_mul(a, b, out)
    assert list(out) == [O.bb_mul(int(x), int(y)) for x, y in zip(a, b)]


def test_bb_polynomial_multiplication(ctx):  # ntt_cross_validation.rs:113-148
    b = sfntt.BbCudaCtGsR4(ctx)
    x = np.array([O.bb_to_monty(1), O.bb_to_monty(2), 0, 0], np.uint32)
    y = np.array([O.bb_to_monty(3), O.bb_to_monty(4), 0, 0], np.uint32)
    b.forward_ntt(x)
    b.forward_ntt(y)
    c = np.zeros(4, np.uint32)
    b.pointwise_mul(x, y, c)
    b.inverse_ntt(c)
    assert [O.bb_from_monty(int(v)) for v in c] == [3, 10, 8, 0]


# ---- batches (src/ntt/babybear/batch.rs:438-505) -------------------------------
@pytest.mark.parametrize("field", [BB, M31])
@pytest.mark.parametrize("log_n,batch", [(1, 5), (4, 3), (8, 64), (10, 7), (12, 2), (13, 1), (14, 16), (20, 3)])
def test_batch_equals_single(ctx, field, log_n, batch):
    b = (sfntt.BbBatchNtt if field == BB else sfntt.CudaCtGsR4)(ctx)
    x = data(field, batch << log_n, 100 + log_n)
    fw, _ = b.forward_ntt_batch_gpu(x, log_n, batch)
    n = 1 << log_n
    for c in range(batch):
        assert np.array_equal(fw[c * n:(c + 1) * n], ofwd(field, x[c * n:(c + 1) * n])), c
    back, _ = b.inverse_ntt_batch_gpu(fw, log_n, batch)
    assert np.array_equal(back, x)
    with pytest.raises(sfntt.InvalidSize):
        b.forward_ntt_batch_gpu(x[:-1], log_n, batch)


@pytest.mark.parametrize("field", [BB, M31])
@pytest.mark.parametrize("log_n,batch", [(8, 4096), (10, 1024), (9, 777)])
def test_many_small_columns(ctx, field, log_n, batch):
    """Lattice-crypto shapes: thousands of 256..1024-point NTTs in one batch
    (sampled columns against the oracle, the whole batch round-trips)."""
    b = (sfntt.BbBatchNtt if field == BB else sfntt.CudaCtGsR4)(ctx)
    x = data(field, batch << log_n, 300 + log_n)
    fw, _ = b.forward_ntt_batch_gpu(x, log_n, batch)
    n = 1 << log_n
    for c in sorted({0, 1, batch // 3, batch // 2 + 5, batch - 2, batch - 1}):
        assert np.array_equal(fw[c * n:(c + 1) * n], ofwd(field, x[c * n:(c + 1) * n])), c
    back, _ = b.inverse_ntt_batch_gpu(fw, log_n, batch)
    assert np.array_equal(back, x)


# ---- coset LDE (src/lde/mod.rs:194-271) ----------------------------------------
@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("log_n,batch,added", [(8, 4, 1), (12, 8, 1), (8, 4, 2), (0, 3, 1), (1, 2, 2), (5, 3, 3),
                                                (13, 2, 1), (14, 3, 2), (16, 4, 1), (18, 2, 1), (11, 5, 4),
                                                (6, 2, 5),
                                                # >= 16 columns: chunk-staged twiddles in the fused expand,
                                                # chunk changes inside a CTA's tile range
                                                (13, 16, 1), (14, 24, 2), (15, 17, 1), (16, 33, 3), (17, 16, 4)])
def test_coset_lde_matches_cpu(ctx, fused, log_n, batch, added):
    lde = sfntt.CosetLdeBatch(ctx, fused=fused)
    x = O.lcg(batch << log_n, 42, O.BB_P, monty=True)
    r = lde.execute(x, log_n, batch, added)
    assert np.array_equal(r.data, O.bb_coset_lde(x, log_n, batch, added, threads=8))


@pytest.mark.parametrize("fused", [True, False])
def test_coset_lde_plonky3_shift(ctx, fused):
    sh = O.bb_to_monty(31)
    x = O.lcg(4 << 14, 7, O.BB_P, monty=True)
    r = sfntt.CosetLdeBatch(ctx, fused=fused).execute(x, 14, 4, 1, shift_monty=sh)
    assert np.array_equal(r.data, O.bb_coset_lde(x, 14, 4, 1, sh, threads=4))


def test_coset_lde_rejects_bad_length(ctx):
    with pytest.raises(sfntt.InvalidSize):
        sfntt.CosetLdeBatch(ctx).execute(np.zeros(100, np.uint32), 8, 4, 1)


@pytest.mark.parametrize("added", [1, 2])
def test_coset_lde_full_size_sampled_columns(ctx, added):
    """2^20 x 256 (the headline shape): every column on the GPU, a sample of
    columns against the oracle, and the low-degree property on all columns."""
    log_n, batch = 20, 256 if added == 1 else 64
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    x = O.lcg(batch << log_n, 2024 + added, O.BB_P, monty=True)
    r = sfntt.CosetLdeBatch(ctx).execute(x, log_n, batch, added)
    for c in (0, 1, batch // 2, batch - 1):
        assert np.array_equal(r.data[c * n_ext:(c + 1) * n_ext],
                              O.bb_coset_lde(x[c * n:(c + 1) * n], log_n, 1, added)), c
    # interpolating the extension gives a polynomial of degree < n on the coset
    coeffs, _ = sfntt.BbBatchNtt(ctx).inverse_ntt_batch_gpu(r.data, log_n + added, batch)
    coeffs = coeffs.reshape(batch, n_ext)
    assert not coeffs[:, n:].any()


def test_m31_lde_matches_composition(ctx, golden):
    meta, arr = golden
    m = sfntt.M31Lde(ctx)
    for case in meta["m31_lde"]:
        r = m.execute(arr[case["input"]], case["log_n"], case["batch"], case["added_bits"])
        assert np.array_equal(r.data, arr[case["output"]])
    # log_n >= 13 runs the fused TMA path (inverse, n^-1, replication, forward in one kernel)
    for (ln, b, ab) in ((12, 3, 1), (13, 2, 1), (14, 2, 2), (16, 2, 1), (17, 1, 3), (15, 3, 4), (20, 2, 1)):
        x = O.lcg(b << ln, ln, O.M31_P)
        assert np.array_equal(m.execute(x, ln, b, ab).data, O.m31_lde(x, ln, b, ab, threads=8)), (ln, b, ab)


def test_m31_lde_full_size_sampled_columns(ctx):
    """2^20 x 128 M31 blow-up: sampled columns against the oracle; the
    inverse of the extension is the input followed by zeros on every column."""
    log_n, batch, added = 20, 128, 1
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    x = O.lcg(batch << log_n, 77, O.M31_P)
    r = sfntt.M31Lde(ctx).execute(x, log_n, batch, added)
    for c in (0, batch // 2 + 1, batch - 1):
        assert np.array_equal(r.data[c * n_ext:(c + 1) * n_ext], O.m31_lde(x[c * n:(c + 1) * n], log_n, 1, added)), c
    m31 = sfntt.CudaCtGsR4(ctx)
    ext, _ = m31.inverse_ntt_batch_gpu(r.data, log_n + added, batch)
    base, _ = m31.inverse_ntt_batch_gpu(x, log_n, batch)
    ext = ext.reshape(batch, n_ext)
    assert not ext[:, n:].any()
    assert np.array_equal(ext[:, :n], base.reshape(batch, n))


@pytest.mark.parametrize("log_n,batch", [(20, 16), (20, 17)])
def test_m31_batch_staged_tile_twiddles(ctx, log_n, batch):
    """M31 12-layer contiguous passes (2^20 columns: 12 + 8 layers) over >= 16
    columns stage each tile's twiddles once for all of its columns (tiles
    column-fastest, a CTA's range crossing tile positions at odd column
    counts): every column against the oracle, and the round trip."""
    b = sfntt.CudaCtGsR4(ctx)
    x = data(M31, batch << log_n, 900 + log_n)
    fw, _ = b.forward_ntt_batch_gpu(x, log_n, batch)
    n = 1 << log_n
    for c in range(batch):
        assert np.array_equal(fw[c * n:(c + 1) * n], O.m31_forward(x[c * n:(c + 1) * n])), c
    back, _ = b.inverse_ntt_batch_gpu(fw, log_n, batch)
    assert np.array_equal(back, x)


def test_m31_lde_staged_odd_columns(ctx):
    """M31 blow-up 2^20 x 17: the staged contiguous passes with tile ranges
    that change position inside a CTA; sampled columns against the oracle."""
    log_n, batch, added = 20, 17, 1
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    x = O.lcg(batch << log_n, 1717, O.M31_P)
    r = sfntt.M31Lde(ctx).execute(x, log_n, batch, added)
    for c in (0, 8, batch - 1):
        assert np.array_equal(r.data[c * n_ext:(c + 1) * n_ext], O.m31_lde(x[c * n:(c + 1) * n], log_n, 1, added)), c


def test_extension_size_cannot_wrap(ctx):
    """log_n + added_bits is range-checked before it is summed in 32 bits:
    an added_bits near 2^32 must not wrap into a small, accepted size."""
    huge = (1 << 32) - 4
    x = O.lcg(1 << 5, 1, O.BB_P, monty=True)
    for lde in (sfntt.CosetLdeBatch(ctx), sfntt.KbCosetLdeBatch(ctx), sfntt.M31Lde(ctx), sfntt.CircleLde(ctx)):
        with pytest.raises(sfntt.InvalidSize):
            lde.execute(x, 5, 1, huge)
    with pytest.raises(sfntt.InvalidSize):
        sfntt.CircleLde(ctx).prepare(5, huge)
    with pytest.raises(sfntt.InvalidSize):
        ctx.prepare_lde(BB, 5, huge)
    import torch
    d = torch.zeros(64, dtype=torch.int32, device="cuda")
    items = [{"field": BB, "log_n": 5, "batch": 1, "added_bits": huge, "d_in": d.data_ptr(), "d_out": d.data_ptr()}]
    with pytest.raises(sfntt.InvalidSize):
        sfntt.LdeBatch(ctx, items).prepare()


@pytest.mark.parametrize("log_n,batch,added", [(21, 2, 1), (22, 1, 1), (21, 1, 2)])
def test_large_lde_multi_pass_layers(ctx, log_n, batch, added):
    """Above 2^20 rows the LDE's outer layer ranges split into contiguous and
    strided passes (BabyBear and M31), and the natural-order form takes the
    bit-reversal route: every column against the oracle."""
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    x = O.lcg(batch << log_n, 60 + log_n, O.BB_P, monty=True)
    r = sfntt.CosetLdeBatch(ctx).execute(x, log_n, batch, added)
    assert np.array_equal(r.data, O.bb_coset_lde(x, log_n, batch, added, threads=8))
    m = O.lcg(batch << log_n, 70 + log_n, O.M31_P)
    assert np.array_equal(sfntt.M31Lde(ctx).execute(m, log_n, batch, added).data,
                          O.m31_lde(m, log_n, batch, added, threads=8))
    if batch == 1 and added == 1:
        rev = lambda bits: np.array([int(format(k, f"0{bits}b")[::-1], 2) for k in range(1 << bits)])
        nat = sfntt.CosetLdeBatch(ctx, natural=True).execute(x[rev(log_n)], log_n, 1, added).data
        assert np.array_equal(nat, r.data[rev(log_n + added)])


@pytest.mark.parametrize("log_n", [13, 14, 15, 17, 18, 19])
def test_m31_batch_staged_any_layer_count(ctx, log_n):
    """M31 contiguous passes of 5..12 layers over >= 16 columns stage each
    tile's per-block twiddles once for all its columns (table order for
    layer counts other than 12): every column against the oracle, and the
    round trip."""
    batch = 16
    b = sfntt.CudaCtGsR4(ctx)
    x = data(M31, batch << log_n, 1900 + log_n)
    fw, _ = b.forward_ntt_batch_gpu(x, log_n, batch)
    n = 1 << log_n
    for c in range(batch):
        assert np.array_equal(fw[c * n:(c + 1) * n], O.m31_forward(x[c * n:(c + 1) * n])), c
    back, _ = b.inverse_ntt_batch_gpu(fw, log_n, batch)
    assert np.array_equal(back, x)


def test_m31_lde_staged_multi_pass(ctx):
    """M31 blow-up 2^21 x 17, 4x: the 13-layer ranges run as a staged 5-layer
    contiguous pass and an 8-layer strided pass; sampled columns against the
    oracle."""
    log_n, batch, added = 21, 17, 2
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    x = O.lcg(batch << log_n, 2121, O.M31_P)
    r = sfntt.M31Lde(ctx).execute(x, log_n, batch, added)
    for c in (0, 9, batch - 1):
        assert np.array_equal(r.data[c * n_ext:(c + 1) * n_ext], O.m31_lde(x[c * n:(c + 1) * n], log_n, 1, added)), c
