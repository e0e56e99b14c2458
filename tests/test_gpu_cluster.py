"""The one-launch cluster NTT (columns of 2^13 .. 2^16 points, one CTA per
2^13-point block of a column, blocks exchanged through distributed shared
memory) against the oracle, bit for bit, for all three fields; the kernel
names recorded by the context show that the cluster kernel ran, and shapes
past one wave of CTAs show the hand-over to the multi-pass engine.
"""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = {
    sfntt.FIELD_BABYBEAR: (sfntt.BbCudaCtGsR4, O.BB_P, True, O.bb_forward, O.bb_inverse),
    sfntt.FIELD_KOALABEAR: (sfntt.KbCudaCtGsR4, O.KB_P, True, O.kb_forward, O.kb_inverse),
    sfntt.FIELD_M31: (sfntt.CudaCtGsR4, O.M31_P, False, O.m31_forward, O.m31_inverse),
}


@pytest.fixture(scope="module")
def ctx():
    return sfntt.default_context(0)


def _kernels(ctx, fn):
    ctx.kernel_timing(True)
    out = fn()
    names = set(ctx.kernel_times())
    ctx.kernel_timing(False)
    return out, names


@pytest.mark.parametrize("field", list(FIELDS))
@pytest.mark.parametrize("log_n,batch", [(13, 1), (14, 1), (15, 1), (16, 1), (13, 5), (14, 3), (15, 7), (16, 2),
                                         (16, 37)])  # 37 x 8 CTAs: exactly two per SM
def test_cluster_ntt_matches_oracle(ctx, field, log_n, batch):
    cls, p, monty, fwd, inv = FIELDS[field]
    b = cls(ctx)
    n = 1 << log_n
    x = O.lcg(batch << log_n, 4000 + 10 * log_n + batch, p, monty=monty)
    fw, names = _kernels(ctx, lambda: b.forward_ntt_batch_gpu(x, log_n, batch)[0])
    assert any("_fwd_cluster" in k for k in names), names
    for c in range(batch):
        assert np.array_equal(fw[c * n:(c + 1) * n], fwd(x[c * n:(c + 1) * n])), c
    back, names = _kernels(ctx, lambda: b.inverse_ntt_batch_gpu(fw, log_n, batch)[0])
    assert any("_inv_cluster" in k for k in names), names
    assert np.array_equal(back, x)
    # the inverse on its own input: the oracle's inverse, not just the round trip
    iv = b.inverse_ntt_batch_gpu(x, log_n, batch)[0]
    for c in (0, batch - 1):
        assert np.array_equal(iv[c * n:(c + 1) * n], inv(x[c * n:(c + 1) * n])), c


@pytest.mark.parametrize("field", [sfntt.FIELD_BABYBEAR, sfntt.FIELD_M31])
def test_past_one_wave_takes_the_pass_engine(ctx, field):
    """38 columns of 2^16 need 304 CTAs: the multi-pass engine runs them, with
    the same results."""
    cls, p, monty, fwd, _ = FIELDS[field]
    log_n, batch, n = 16, 38, 1 << 16
    x = O.lcg(batch << log_n, 77, p, monty=monty)
    fw, names = _kernels(ctx, lambda: cls(ctx).forward_ntt_batch_gpu(x, log_n, batch)[0])
    assert not any("cluster" in k for k in names), names
    for c in (0, batch - 1):
        assert np.array_equal(fw[c * n:(c + 1) * n], fwd(x[c * n:(c + 1) * n])), c


def test_single_ntt_entry_points_use_the_cluster(ctx):
    """The single-column calls (forward_ntt_gpu / inverse_ntt_gpu) reach the
    same kernel: the reference's BabyBear polynomial product
    (ntt_cross_validation.rs:113-148) at 2^14 points."""
    b = sfntt.BbCudaCtGsR4(ctx)
    log_n = 14
    a = np.zeros(1 << log_n, np.uint32)
    c = np.zeros(1 << log_n, np.uint32)
    a[:2] = [O.bb_to_monty(v) for v in (1, 2)]
    c[:2] = [O.bb_to_monty(v) for v in (3, 4)]
    (fa, names) = _kernels(ctx, lambda: b.forward_ntt_gpu(a, log_n)[0])
    assert any("_fwd_cluster" in k for k in names), names
    fc = b.forward_ntt_gpu(c, log_n)[0]
    prod = np.empty_like(fa)
    b.pointwise_mul(fa, fc, prod)
    out, names = _kernels(ctx, lambda: b.inverse_ntt_gpu(prod, log_n)[0])
    assert any("_inv_cluster" in k for k in names), names
    assert [O.bb_from_monty(int(v)) for v in out[:4]] == [3, 10, 8, 0] and not out[4:].any()


def test_no_cluster_switch_keeps_the_passes(tmp_path):
    """SFNTT_NO_CLUSTER=1 (read at context creation) runs 2^13..2^16-point
    columns as two passes: same results, no cluster kernel."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    script = tmp_path / "no_cluster.py"
    script.write_text(
        "import sys\n"
        f"sys.path[:0] = [{str(root)!r}, {str(root / 'small-field-metal-ntt_b200')!r}]\n"
        "import numpy as np, sfntt\n"
        "from oracle import oracle as O\n"
        "ctx = sfntt.Context(0)\n"
        "b = sfntt.CudaCtGsR4(ctx)\n"
        "x = O.lcg(3 << 15, 5, O.M31_P)\n"
        "ctx.kernel_timing(True)\n"
        "fw = b.forward_ntt_batch_gpu(x, 15, 3)[0]\n"
        "names = set(ctx.kernel_times())\n"
        "assert not any('cluster' in k for k in names), names\n"
        "n = 1 << 15\n"
        "assert all(np.array_equal(fw[c * n:(c + 1) * n], O.m31_forward(x[c * n:(c + 1) * n])) for c in range(3))\n"
        "assert np.array_equal(b.inverse_ntt_batch_gpu(fw, 15, 3)[0], x)\n"
        "print('ok')\n")
    env = dict(os.environ, SFNTT_NO_CLUSTER="1")
    r = subprocess.run([sys.executable, str(script)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
