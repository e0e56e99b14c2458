"""Uneven batches in one graph launch (both fields, uneven sizes and blow-ups).

Every item must give the same result alone (the oracle: the reference's
coset_lde_batch_cpu for BabyBear, the inverse/zero-pad/forward composition for
M31), in the plain per-item loop, in the captured CUDA graph and under any
autotuned plan.
"""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _alloc(items, seed):
    import torch
    bufs = []
    for k, it in enumerate(items):
        p = O.BB_P if it["field"] == sfntt.FIELD_BABYBEAR else O.M31_P
        x = O.lcg(it["batch"] << it["log_n"], seed + k, p, monty=(it["field"] == sfntt.FIELD_BABYBEAR))
        d_in = torch.from_numpy(x.view(np.int32).copy()).cuda()
        d_out = torch.zeros(it["batch"] << (it["log_n"] + it["added_bits"]), dtype=torch.int32, device="cuda")
        it["d_in"], it["d_out"] = d_in.data_ptr(), d_out.data_ptr()
        bufs.append((x, d_in, d_out))
    return bufs


def _oracle(it, x):
    if it["field"] == sfntt.FIELD_BABYBEAR:
        return O.bb_coset_lde(x, it["log_n"], it["batch"], it["added_bits"], threads=8)
    return O.m31_lde(x, it["log_n"], it["batch"], it["added_bits"], threads=8)


@pytest.fixture(scope="module")
def ctx():
    return sfntt.Context(0)


def test_uneven_batch_plain_graph_tuned_match_oracle(ctx):
    import torch
    items = sfntt.uneven_workload(24, seed=7, log_n_range=(1, 15), cols_range=(1, 9))
    bufs = _alloc(items, 100)
    batch = sfntt.LdeBatch(ctx, items)
    batch.prepare()
    batch.run()
    torch.cuda.synchronize()
    plain = [b[2].cpu().numpy().view(np.uint32).copy() for b in bufs]
    for it, (x, _, _), got in zip(items, bufs, plain):
        assert np.array_equal(got, _oracle(it, x)), it
    for b in bufs:
        b[2].zero_()
    g = batch.graph(lanes=4)
    assert g.kernel_count() > 0
    g.launch()
    g.launch()  # replay is idempotent
    torch.cuda.synchronize()
    for b, ref in zip(bufs, plain):
        assert np.array_equal(b[2].cpu().numpy().view(np.uint32), ref)
    batch.autotune(reps=1)
    plans = {batch.plan_of(i) for i in range(len(items))}
    engines = {sfntt.PLAN_TMA, sfntt.PLAN_TMA_FOUR_STEP}
    valid = {e | f for e in engines for f in (0, sfntt.PLAN_SPLIT12, sfntt.PLAN_ONE_CTA,
                                              sfntt.PLAN_SPLIT12 | sfntt.PLAN_ONE_CTA)} | {sfntt.PLAN_TILE}
    assert plans <= valid and plans
    for b in bufs:
        b[2].zero_()
    batch.run()
    torch.cuda.synchronize()
    for b, ref in zip(bufs, plain):
        assert np.array_equal(b[2].cpu().numpy().view(np.uint32), ref)
    g.close()


@pytest.mark.parametrize("plan", [sfntt.PLAN_TMA, sfntt.PLAN_TMA_FOUR_STEP, sfntt.PLAN_TILE,
                                  sfntt.PLAN_TMA | sfntt.PLAN_SPLIT12, sfntt.PLAN_TMA_FOUR_STEP | sfntt.PLAN_SPLIT12,
                                  sfntt.PLAN_TMA | sfntt.PLAN_ONE_CTA,
                                  sfntt.PLAN_TMA_FOUR_STEP | sfntt.PLAN_SPLIT12 | sfntt.PLAN_ONE_CTA])
def test_every_plan_is_exact(ctx, plan):
    """Every engine and knob, on shapes where the layer split differs (a
    layer range of 13..14 layers: 12 + 1..2 against 5..6 + 8)."""
    import torch
    items = [{"field": sfntt.FIELD_BABYBEAR, "log_n": 14, "batch": 3, "added_bits": 2, "plan": plan},
             {"field": sfntt.FIELD_BABYBEAR, "log_n": 16, "batch": 2, "added_bits": 0, "plan": plan},
             {"field": sfntt.FIELD_M31, "log_n": 15, "batch": 2, "added_bits": 1, "plan": plan},
             {"field": sfntt.FIELD_BABYBEAR, "log_n": 21, "batch": 1, "added_bits": 1, "plan": plan},
             {"field": sfntt.FIELD_BABYBEAR, "log_n": 22, "batch": 1, "added_bits": 0, "plan": plan},
             {"field": sfntt.FIELD_M31, "log_n": 22, "batch": 1, "added_bits": 1, "plan": plan}]
    bufs = _alloc(items, 900 + plan)
    with pytest.raises(sfntt.InvalidArgument):
        sfntt.LdeBatch(ctx, [dict(items[0], plan=16)]).run()
    batch = sfntt.LdeBatch(ctx, items)
    batch.prepare()
    batch.run()
    torch.cuda.synchronize()
    for it, (x, _, d_out) in zip(items, bufs):
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), _oracle(it, x)), it


def test_tune_table_roundtrip(ctx, tmp_path):
    items = [{"field": sfntt.FIELD_BABYBEAR, "log_n": 13, "batch": 2, "added_bits": 1}]
    _alloc(items, 5)
    b = sfntt.LdeBatch(ctx, items)
    b.autotune(reps=1)
    plan = b.plan_of(0)
    path = tmp_path / "tune.txt"
    sfntt.tune_save(ctx, path)
    fresh = sfntt.Context(0)
    sfntt.tune_load(fresh, path)
    assert sfntt.LdeBatch(fresh, items).plan_of(0) == plan
    fresh.close()


def test_persistent_phases_match_oracle(ctx):
    """Items of both fields, 2^12..2^17 points, 1..40 columns, blow-ups
    1/2/4/16: the eligible ones (2^13..2^20 points) run in the three
    persistent phase launches over a device work list (BabyBear items with
    >= 16 columns on staged twiddle chunks), the others per item beside them;
    every output equals the oracle, on two replays of the graph."""
    import torch
    items = sfntt.uneven_workload(20, seed=31, log_n_range=(12, 17), cols_range=(1, 40))
    items += [{"field": sfntt.FIELD_BABYBEAR, "log_n": 14, "batch": 17, "added_bits": 4},
              {"field": sfntt.FIELD_M31, "log_n": 13, "batch": 33, "added_bits": 2},
              {"field": sfntt.FIELD_BABYBEAR, "log_n": 13, "batch": 16, "added_bits": 0}]
    bufs = _alloc(items, 4100)
    batch = sfntt.LdeBatch(ctx, items)
    batch.prepare()
    g = batch.persistent_graph(lanes=4)
    assert g.kernel_count() > 0
    for rep in range(2):
        for b in bufs:
            b[2].zero_()
        g.launch()
        torch.cuda.synchronize()
        assert ctx.check_device_error() == 0
        for it, (x, _, d_out) in zip(items, bufs):
            assert np.array_equal(d_out.cpu().numpy().view(np.uint32), _oracle(it, x)), (rep, it)
    g.close()


def test_persistent_phases_large_items():
    """2^20- and 2^21-point items of both fields with many columns (the staged
    BabyBear expansion, 12- and 13-layer contiguous passes): sampled columns
    against the oracle and the whole output against the per-item launches."""
    import os
    import torch
    # a context whose work list takes items of any size (the default leaves
    # items of more than 16 tiles per SM to their own launches)
    old = os.environ.get("SFNTT_WORKLIST_TILES")
    os.environ["SFNTT_WORKLIST_TILES"] = "0"
    try:
        ctx = sfntt.Context(0)
    finally:
        if old is None:
            del os.environ["SFNTT_WORKLIST_TILES"]
        else:
            os.environ["SFNTT_WORKLIST_TILES"] = old
    items = [{"field": sfntt.FIELD_BABYBEAR, "log_n": 20, "batch": 24, "added_bits": 1},
             {"field": sfntt.FIELD_M31, "log_n": 19, "batch": 20, "added_bits": 2},
             {"field": sfntt.FIELD_BABYBEAR, "log_n": 18, "batch": 5, "added_bits": 2},
             # 2^21: 13-layer contiguous phases
             {"field": sfntt.FIELD_M31, "log_n": 21, "batch": 18, "added_bits": 1},
             {"field": sfntt.FIELD_BABYBEAR, "log_n": 21, "batch": 17, "added_bits": 1}]
    bufs = _alloc(items, 5100)
    batch = sfntt.LdeBatch(ctx, items)
    batch.prepare()
    batch.run()
    torch.cuda.synchronize()
    plain = [b[2].clone() for b in bufs]
    for b in bufs:
        b[2].zero_()
    g = batch.persistent_graph(lanes=2)
    g.launch()
    torch.cuda.synchronize()
    for it, (x, _, d_out), ref in zip(items, bufs, plain):
        assert torch.equal(d_out, ref), it
        n, n_ext = 1 << it["log_n"], 1 << (it["log_n"] + it["added_bits"])
        got = d_out.cpu().numpy().view(np.uint32)
        for c in (0, it["batch"] - 1):
            sub = dict(it, batch=1)
            assert np.array_equal(got[c * n_ext:(c + 1) * n_ext], _oracle(sub, x[c * n:(c + 1) * n])), (it, c)
    g.close()
