"""Contiguous passes with whole-tile copies, against the oracle.

By default the 8- and 12-layer contiguous passes run two independent
half-tile pipelines per CTA; with SFNTT_HALVES=0 (read when a context is
created, hence the child process) they move whole tiles -- for the
row-permuted layouts of 8-, 11- and 12-layer passes, two half-tile copies per
tile into one buffer.  The child checks NTTs of both fields (src/ntt/babybear/
cpu_reference.rs:34-103, src/ntt/m31/cpu_reference.rs:50-120) and the fused
coset LDE (src/lde/mod.rs:127-176) bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import numpy as np
import sfntt
from oracle import oracle as O

ctx = sfntt.default_context(0)
bb, m31 = sfntt.BbCudaCtGsR4(ctx), sfntt.CudaCtGsR4(ctx)
for log_n in (13, 16, 19, 20, 21, 24):
    x = O.lcg(1 << log_n, 900 + log_n, O.BB_P, monty=True)
    fw, _ = bb.forward_ntt_gpu(x, log_n)
    assert np.array_equal(fw, O.bb_forward(x)), ("bb fwd", log_n)
    iv, _ = bb.inverse_ntt_gpu(x, log_n)
    assert np.array_equal(iv, O.bb_inverse(x)), ("bb inv", log_n)
for log_n in (13, 17, 20, 21):
    x = O.lcg(1 << log_n, 700 + log_n, O.M31_P)
    fw, _ = m31.forward_ntt_gpu(x, log_n)
    assert np.array_equal(fw, O.m31_forward(x)), ("m31 fwd", log_n)
    iv, _ = m31.inverse_ntt_gpu(x, log_n)
    assert np.array_equal(iv, O.m31_inverse(x)), ("m31 inv", log_n)
for log_n, batch, added in ((13, 16, 1), (16, 8, 2), (20, 2, 1)):
    x = O.lcg(batch << log_n, 42 + log_n, O.BB_P, monty=True)
    r = sfntt.CosetLdeBatch(ctx).execute(x, log_n, batch, added)
    assert np.array_equal(r.data, O.bb_coset_lde(x, log_n, batch, added, threads=8)), ("lde", log_n)
print("whole tiles ok")
"""


def test_whole_tile_passes_match_oracle():
    env = dict(os.environ, SFNTT_HALVES="0",
               PYTHONPATH=os.pathsep.join([str(ROOT), str(ROOT / "small-field-metal-ntt_b200"),
                                           os.environ.get("PYTHONPATH", "")]))
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0 and "whole tiles ok" in r.stdout, (r.stdout[-2000:], r.stderr[-4000:])
