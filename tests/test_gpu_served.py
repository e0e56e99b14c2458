"""Serving with continuous batching (sfntt_server_*, sfntt_serve_trace).

Requests of both fields and uneven sizes are admitted as slots and arena
space free up; every request must give the same output in the mix as alone
(the plain per-request call) and as the oracle (the reference's
coset_lde_batch_cpu for BabyBear, inverse/zero-pad/forward for M31).
"""
from __future__ import annotations

import numpy as np
import pytest

import sfntt
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return sfntt.Context(0)


def _input(it, seed):
    bb = it["field"] == sfntt.FIELD_BABYBEAR
    return O.lcg(it["batch"] << it["log_n"], seed, O.BB_P if bb else O.M31_P, monty=bb)


def _oracle(it, x):
    if it["field"] == sfntt.FIELD_BABYBEAR:
        return O.bb_coset_lde(x, it["log_n"], it["batch"], it["added_bits"], threads=8)
    return O.m31_lde(x, it["log_n"], it["batch"], it["added_bits"], threads=8)


def _alone(ctx, it, d_in):
    """The plain drop-in call for one request, on its own output buffer."""
    import torch
    out = torch.zeros(it["batch"] << (it["log_n"] + it["added_bits"]), dtype=torch.int32, device="cuda")
    if it["field"] == sfntt.FIELD_BABYBEAR:
        sfntt.CosetLdeBatch(ctx).execute_dev(d_in.data_ptr(), out.data_ptr(), it["log_n"], it["batch"],
                                             it["added_bits"])
    else:
        sfntt.M31Lde(ctx).execute_dev(d_in.data_ptr(), out.data_ptr(), it["log_n"], it["batch"], it["added_bits"])
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32).copy()


def _mix(n, seed):
    reqs = sfntt.uneven_workload(n, seed=seed, log_n_range=(1, 15), cols_range=(1, 9))
    # BabyBear outside the fused range (runs alone on the context scratch)
    reqs.insert(5, {"field": sfntt.FIELD_BABYBEAR, "log_n": 6, "batch": 3, "added_bits": 5})
    reqs.insert(9, {"field": sfntt.FIELD_BABYBEAR, "log_n": 0, "batch": 4, "added_bits": 2})
    return reqs


def test_each_result_same_alone_and_in_the_mix(ctx):
    import torch
    reqs = _mix(28, seed=11)
    xs = [_input(it, 500 + i) for i, it in enumerate(reqs)]
    d_ins = [torch.from_numpy(x.view(np.int32).copy()).cuda() for x in xs]
    for it, d in zip(reqs, d_ins):
        it["d_in"] = d.data_ptr()
    # small budget: admission has to wait for arena space, slots overlap
    budget = 3 * max(it["batch"] << (it["log_n"] + it["added_bits"]) for it in reqs) * 4
    srv = sfntt.Server(ctx, budget_bytes=budget, slots=4)
    tickets, got = {}, {}
    for i, it in enumerate(reqs):  # arrivals in bursts while earlier ones run
        tickets[srv.submit(it)] = i
        if i % 3 == 2:
            for t in srv.poll():
                it_t = reqs[tickets[t]]
                got[tickets[t]] = srv.result(t, it_t["batch"] << (it_t["log_n"] + it_t["added_bits"])).cpu().numpy() \
                    .view(np.uint32).copy()
                srv.release(t)
    while len(got) < len(reqs):
        for t in srv.poll():
            it_t = reqs[tickets[t]]
            got[tickets[t]] = srv.result(t, it_t["batch"] << (it_t["log_n"] + it_t["added_bits"])).cpu().numpy() \
                .view(np.uint32).copy()
            srv.release(t)
    assert srv.pending() == 0
    srv.close()
    for i, (it, x, d) in enumerate(zip(reqs, xs, d_ins)):
        alone = _alone(ctx, it, d)
        assert np.array_equal(got[i], alone), (i, it)
        assert np.array_equal(alone, _oracle(it, x)), (i, it)


def test_host_requests_match_oracle(ctx):
    reqs = _mix(12, seed=12)
    srv = sfntt.Server(ctx, budget_bytes=64 << 20, slots=3)
    outs = {}
    for i, it in enumerate(reqs):
        x = _input(it, 900 + i)
        t, out = srv.submit_host(it, x)
        outs[t] = (i, x, out)
    done = set()
    while len(done) < len(reqs):
        for t in srv.poll():
            done.add(t)
            srv.release(t)
    for t, (i, x, out) in outs.items():
        assert np.array_equal(out, _oracle(reqs[i], x)), (i, reqs[i])
    srv.close()


def test_request_over_budget_is_refused(ctx):
    import torch
    d = torch.zeros(1 << 12, dtype=torch.int32, device="cuda")
    srv = sfntt.Server(ctx, budget_bytes=1 << 16, slots=2)
    it = {"field": sfntt.FIELD_BABYBEAR, "log_n": 12, "batch": 1, "added_bits": 4, "d_in": d.data_ptr()}
    with pytest.raises(sfntt.BufferAllocFailed):
        srv.submit(it)
    it["added_bits"] = 1
    t = srv.submit(it)
    while not srv.poll():
        pass
    srv.release(t)
    with pytest.raises(sfntt.InvalidArgument):
        srv.release(t)
    srv.close()


@pytest.mark.parametrize("slots", [1, 4])
def test_trace_replay_host_outputs_exact(ctx, slots):
    reqs, arrivals = sfntt.served_workload(16, rate=2000.0, seed=5, cols_range=(1, 4),
                                           log_n_weights={10: 1, 12: 1, 14: 2, 15: 1})
    host = []
    for i, it in enumerate(reqs):
        x = _input(it, 1300 + i)
        host.append((x, np.zeros(it["batch"] << (it["log_n"] + it["added_bits"]), dtype=np.uint32)))
    lat, makespan = sfntt.serve_trace(ctx, reqs, arrivals, slots=slots, budget_bytes=32 << 20, host=host)
    assert makespan > 0 and np.all(lat > 0) and np.all(np.isfinite(lat))
    assert makespan >= arrivals[-1]
    for it, (x, out) in zip(reqs, host):
        assert np.array_equal(out, _oracle(it, x)), it


def test_trace_replay_device_inputs(ctx):
    import torch
    reqs, arrivals = sfntt.served_workload(24, rate=500.0, seed=6, cols_range=(1, 8),
                                           log_n_weights={13: 1, 14: 2, 16: 1})
    pool = torch.randint(0, O.BB_P, (8 << 16,), dtype=torch.int64, device="cuda").to(torch.int32)
    for it in reqs:
        it["d_in"] = pool.data_ptr()  # inputs are slices of one resident pool
    lat_plain, mk_plain = sfntt.serve_trace(ctx, reqs, arrivals, slots=1, budget_bytes=256 << 20)
    lat_srv, mk_srv = sfntt.serve_trace(ctx, reqs, arrivals, slots=8, budget_bytes=256 << 20)
    for lat in (lat_plain, lat_srv):
        assert np.all(lat > 0) and np.all(np.isfinite(lat))
    assert mk_plain >= arrivals[-1] and mk_srv >= arrivals[-1]


def _small_same_shape_mix(seed):
    """Requests of three shapes (both fields), interleaved, small enough that
    several share the GPU: packing candidates."""
    rng = np.random.default_rng(seed)
    shapes = [(sfntt.FIELD_BABYBEAR, 13, 1), (sfntt.FIELD_M31, 14, 2), (sfntt.FIELD_BABYBEAR, 12, 2)]
    reqs = []
    for i in range(24):
        f, ln, ab = shapes[i % 3]
        reqs.append({"field": f, "log_n": ln, "batch": int(rng.integers(1, 6)), "added_bits": ab})
    return reqs


def test_packed_requests_same_alone_and_in_one_launch(ctx):
    """With packing, queued requests of one shape run as the columns of one
    batch: every request's output equals its plain drop-in call and the
    oracle, device and host requests mixed, and the launches are fewer than
    the requests."""
    import torch
    reqs = _small_same_shape_mix(3)
    xs = [_input(it, 2100 + i) for i, it in enumerate(reqs)]
    d_ins = [torch.from_numpy(x.view(np.int32).copy()).cuda() for x in xs]
    srv = sfntt.Server(ctx, budget_bytes=512 << 20, slots=2)
    srv.set_packing(16)
    tickets, host_out = {}, {}
    for i, (it, d) in enumerate(zip(reqs, d_ins)):
        if i % 4 == 3:  # every fourth request comes from the host
            t, out = srv.submit_host(it, xs[i])
            host_out[i] = out
        else:
            it["d_in"] = d.data_ptr()
            t = srv.submit(it)
        tickets[t] = i
    got = {}
    while len(got) < len(reqs):
        for t in srv.poll():
            i = tickets[t]
            it = reqs[i]
            if i in host_out:
                got[i] = host_out[i]
            else:
                got[i] = srv.result(t, it["batch"] << (it["log_n"] + it["added_bits"])).cpu().numpy() \
                    .view(np.uint32).copy()
            srv.release(t)
    launches = srv.launches()
    assert srv.pending() == 0
    srv.close()
    assert launches < len(reqs), launches
    for i, (it, x, d) in enumerate(zip(reqs, xs, d_ins)):
        alone = _alone(ctx, it, d)
        assert np.array_equal(got[i], alone), (i, it)
        assert np.array_equal(alone, _oracle(it, x)), (i, it)


@pytest.mark.parametrize("max_pack", [1, 8])
def test_trace_replay_packed_host_outputs_exact(ctx, max_pack):
    reqs, arrivals = sfntt.served_workload(32, rate=20000.0, seed=8, cols_range=(1, 4),
                                           log_n_weights={13: 1, 14: 1})
    host = []
    for i, it in enumerate(reqs):
        x = _input(it, 1700 + i)
        host.append((x, np.zeros(it["batch"] << (it["log_n"] + it["added_bits"]), dtype=np.uint32)))
    stats = {}
    lat, makespan = sfntt.serve_trace(ctx, reqs, arrivals, slots=4, budget_bytes=256 << 20, host=host,
                                      max_pack=max_pack, stats=stats)
    assert np.all(lat > 0) and np.all(np.isfinite(lat))
    assert stats["launches"] <= len(reqs)
    if max_pack == 1:
        assert stats["launches"] == len(reqs)
    for it, (x, out) in zip(reqs, host):
        assert np.array_equal(out, _oracle(it, x)), it
