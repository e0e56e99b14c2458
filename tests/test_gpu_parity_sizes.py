"""GPU parity on the configured and timed shapes, against the oracle.

* BabyBear forward and inverse at every log n from 10 to 24 (the single-column
  sweep of the reference's CPU path, src/ntt/babybear/cpu_reference.rs:34-103),
  and M31 at every log n from 17 to 24 (src/ntt/m31/cpu_reference.rs:50-120);
* BabyBear canonical <-> Montgomery conversion on the device
  (BabyBear::to_monty / from_monty, src/field/babybear.rs:54-65), through both
  C-ABI entry points;
* the benchmark's own configuration: 2^20 rows x 256 columns, 2x blow-up,
  coset shift g = 31 (shift_monty = to_monty(31)), canonical inputs converted
  to Montgomery form on the device -- sampled columns bit for bit against the
  oracle's coset_lde_batch_cpu (src/lde/mod.rs:127-176 with the shift
  replaced), the low-degree property on every column.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import sfntt
from sfntt import _ffi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

BB, M31 = sfntt.FIELD_BABYBEAR, sfntt.FIELD_M31


@pytest.fixture(scope="module")
def ctx():
    return sfntt.default_context(0)


@pytest.mark.parametrize("log_n", list(range(10, 25)))
def test_bb_forward_inverse_every_size(ctx, log_n):
    b = sfntt.BbCudaCtGsR4(ctx)
    x = O.lcg(1 << log_n, 4242 + log_n, O.BB_P, monty=True)
    fw, _ = b.forward_ntt_gpu(x, log_n)
    assert np.array_equal(fw, O.bb_forward(x)), log_n
    iv, _ = b.inverse_ntt_gpu(x, log_n)
    assert np.array_equal(iv, O.bb_inverse(x)), log_n
    back, _ = b.inverse_ntt_gpu(fw, log_n)
    assert np.array_equal(back, x), log_n


@pytest.mark.parametrize("log_n", [19, 21, 22, 23, 24])
def test_m31_forward_inverse_large_sizes(ctx, log_n):
    b = sfntt.CudaCtGsR4(ctx)
    x = O.lcg(1 << log_n, 515 + log_n, O.M31_P)
    fw, _ = b.forward_ntt_gpu(x, log_n)
    assert np.array_equal(fw, O.m31_forward(x)), log_n
    iv, _ = b.inverse_ntt_gpu(x, log_n)
    assert np.array_equal(iv, O.m31_inverse(x)), log_n


def _bb_conversion_inputs() -> np.ndarray:
    p = O.BB_P
    edges = np.array([0, 1, 2, 31, p - 2, p - 1, (1 << 27), (1 << 30) - 1, 1 << 30], np.uint32)
    return np.concatenate([edges, O.lcg(100_003, 54, p)])


@pytest.mark.parametrize("entry", ["bb", "generic"])
def test_bb_monty_conversion_on_device(ctx, entry):
    import torch
    L = _ffi.lib()
    v = _bb_conversion_inputs()
    d = torch.from_numpy(v.view(np.int32).copy()).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    if entry == "bb":
        to = lambda: L.sfntt_bb_to_monty_dev(ctx.handle, d.data_ptr(), v.size, stream)
        back = lambda: L.sfntt_bb_from_monty_dev(ctx.handle, d.data_ptr(), v.size, stream)
    else:
        to = lambda: L.sfntt_to_monty_dev(ctx.handle, BB, d.data_ptr(), v.size, stream)
        back = lambda: L.sfntt_from_monty_dev(ctx.handle, BB, d.data_ptr(), v.size, stream)
    assert to() == 0, L.sfntt_last_error(ctx.handle)
    torch.cuda.synchronize()
    m = d.cpu().numpy().view(np.uint32)
    assert np.array_equal(m, O.bb_to_monty_array(v))
    assert back() == 0, L.sfntt_last_error(ctx.handle)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), v)
    # from_monty of arbitrary Montgomery words (not produced by to_monty)
    w = O.lcg(4099, 77, O.BB_P)
    d2 = torch.from_numpy(w.view(np.int32).copy()).cuda()
    assert L.sfntt_bb_from_monty_dev(ctx.handle, d2.data_ptr(), w.size, stream) == 0
    torch.cuda.synchronize()
    assert np.array_equal(d2.cpu().numpy().view(np.uint32), O.bb_from_monty_array(w))


def test_bench_configuration_full_size(ctx):
    """The timed configuration exactly: 2^20 x 256, 2x, g = 31, the input
    drawn as the benchmark draws it (seeded uniform canonical values on the
    device, converted to Montgomery form there) and the LDE called through
    the same device entry point."""
    import torch
    log_n, batch, added = 20, 256, 1
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    shift = (31 << 32) % O.BB_P
    assert shift == O.bb_to_monty(31)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234)
    x = torch.randint(0, O.BB_P, (batch * n,), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    out = torch.empty(batch * n_ext, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    sfntt.convert_monty_dev(ctx, BB, x.data_ptr(), x.numel(), to_monty=True, stream=stream)
    sfntt.CosetLdeBatch(ctx).execute_dev(x.data_ptr(), out.data_ptr(), log_n, batch, added, shift_monty=shift,
                                         stream=stream)
    torch.cuda.synchronize()
    cols = (0, 1, 37, 100, 128, 200, 254, 255)
    xin = x.view(batch, n)
    got = out.view(batch, n_ext)
    for c in cols:
        col = xin[c].cpu().numpy().view(np.uint32).copy()
        want = O.bb_coset_lde(col, log_n, 1, added, shift_monty=shift)
        assert np.array_equal(got[c].cpu().numpy().view(np.uint32), want), c
    # low degree on every column: interpolating the 2^21 evaluations (an
    # inverse NTT of each extended column, in place on the device) leaves the
    # upper half of the coefficients zero
    assert torch.all((out >= 0) & (out < O.BB_P)).item()
    sfntt.BbCudaCtGsR4(ctx).inverse_dev(out.data_ptr(), log_n + added, batch, stream=stream)
    torch.cuda.synchronize()
    assert not got[:, n:].any().item()
    # ... and the lower half is the input's coefficients times shift^i
    coeffs = x.clone()
    sfntt.BbCudaCtGsR4(ctx).inverse_dev(coeffs.data_ptr(), log_n, batch, stream=stream)
    torch.cuda.synchronize()
    for c in (0, 255):
        lo = got[c, :n].cpu().numpy().view(np.uint32)
        base = coeffs.view(batch, n)[c].cpu().numpy().view(np.uint32)
        for i in (0, 1, 2, 3, 1000, n - 1):
            sh_i = O.bb_to_monty(pow(31, int(i), O.BB_P))
            assert int(lo[i]) == O.bb_mul(int(base[i]), sh_i), (c, i)


# ---- 13-layer contiguous passes: 2^13 and 2^21 columns (one contiguous pass
# of 13 layers, plus one 8-layer strided pass at 2^21), LDEs whose inverse and
# forward low layers are 13 (log n = 21) ----------------------------------
def _m31_batch(fn, x, log_n, batch):
    n = 1 << log_n
    return np.concatenate([fn(x[c * n:(c + 1) * n]) for c in range(batch)])


@pytest.mark.parametrize("log_n,batch", [(13, 3), (21, 2), (14, 160), (22, 2)])
def test_thirteen_layer_batches(ctx, log_n, batch):
    """13- and 14-layer contiguous passes: 2^13 and 2^21 (13 + 8), 2^14 past
    one cluster wave and 2^22 (14 + 8: the 2^14-word tiles of 1024 threads)."""
    import torch
    n = 1 << log_n
    xb = O.lcg(batch * n, 1300 + log_n, O.BB_P, monty=True)
    xm = O.lcg(batch * n, 1400 + log_n, O.M31_P)
    stream = torch.cuda.current_stream().cuda_stream
    for eng, x, fwd, inv in ((sfntt.BbCudaCtGsR4(ctx), xb, lambda v: O.bb_forward_batch(v, log_n, batch, threads=8),
                              lambda v: O.bb_inverse_batch(v, log_n, batch, threads=8)),
                             (sfntt.CudaCtGsR4(ctx), xm, lambda v: _m31_batch(O.m31_forward, v, log_n, batch),
                              lambda v: _m31_batch(O.m31_inverse, v, log_n, batch))):
        d = torch.from_numpy(x.view(np.int32).copy()).cuda()
        eng.forward_dev(d.data_ptr(), log_n, batch, stream=stream)
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32), fwd(x)), log_n
        d.copy_(torch.from_numpy(x.view(np.int32).copy()))
        eng.inverse_dev(d.data_ptr(), log_n, batch, stream=stream)
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32), inv(x)), log_n


@pytest.mark.parametrize("log_n,batch", [(21, 2), (21, 16), (22, 2), (22, 16)])
def test_lde_log_n_21_22(ctx, log_n, batch):
    """BabyBear coset LDE and M31 blow-up at 2^21 and 2^22 (low layers: one
    13- or 14-layer contiguous pass each way); 16 columns take the M31
    staged-twiddle passes at 2^21 (the 14-layer pass reads them from L2)."""
    added = 1
    xb = O.lcg(batch << log_n, 2100 + batch, O.BB_P, monty=True)
    r = sfntt.CosetLdeBatch(ctx).execute(xb, log_n, batch, added)
    assert np.array_equal(r.data, O.bb_coset_lde(xb, log_n, batch, added, threads=8))
    xm = O.lcg(batch << log_n, 2200 + batch, O.M31_P)
    r = sfntt.M31Lde(ctx).execute(xm, log_n, batch, added)
    assert np.array_equal(r.data, O.m31_lde(xm, log_n, batch, added, threads=8))
