#!/usr/bin/env python3
"""Benchmark of the BabyBear coset LDE, 2^20 rows x 256 columns, 2x blow-up.

This is the reference's headline number (README.md:58: 821 ms on an Apple M3
GPU, timed commit -> wait).  One step = one full LDE of 256 columns
(iDFT -> n^-1 -> zero-pad -> coset shift -> DFT), inputs resident in HBM:
1 GiB in, 2 GiB out, so every step streams more than the 126 MB L2.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU runs (torchrun, one rank per GPU) are weak-scaled replicas: every
rank runs its own 256-column LDE with no data-path collective; `value` is the
job's time per LDE (slowest rank's step time / N).

`--impl reference` times the reference's CPU implementation of the path (the
C restatement in oracle/, all host threads, a bounded sample of columns per
step scaled to 256 columns).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "small-field-metal-ntt_b200"))
sys.path.insert(0, str(ROOT))

BB_P = 2013265921
KB_P = 2130706433  # KoalaBear, 2^31 - 2^24 + 1
METRIC = "BabyBear coset LDE 2^20x256 2x"
PUBLISHED_MS = 821.0  # the reference's README.md:58 (Apple M3, Metal)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--log-n", type=int, default=20)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--added-bits", type=int, default=1)
    ap.add_argument("--mode", default="fused", choices=["fused", "unfused"])
    ap.add_argument("--natural", action="store_true",
                    help="BabyBear / KoalaBear LDE in the natural-order convention (Plonky3's coset_lde_batch rows)")
    ap.add_argument("--field", default="bb", choices=["bb", "m31", "kb"],
                    help="bb: the BabyBear coset LDE (the headline); m31: the M31 blow-up of the same shape; "
                         "kb: the KoalaBear coset LDE of the same shape")
    ap.add_argument("--shift", default="31", choices=["31", "reference"],
                    help="coset shift: the multiplicative generator (31 for BabyBear, 3 for KoalaBear) or the "
                         "reference's default two_adic_generator(log_n_ext + 1); the cost is the same")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--rates", default="50,100,200,500,1000,2000", help="served stream: arrival rates, req/s")
    ap.add_argument("--requests", type=int, default=120, help="served stream: requests per rate")
    ap.add_argument("--slots", type=int, default=8, help="served stream: concurrent request slots")
    ap.add_argument("--pack", type=int, default=32, help="served stream: most same-shape requests per launch")
    ap.add_argument("--budget-gb", type=float, default=64.0, help="served stream: HBM admission budget")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch comparison in the LDE line")
    ap.add_argument("--workload", default="lde", choices=["lde", "uneven", "served", "table", "ntt", "layout"],
                    help="lde: the headline LDE (default); uneven: 64 mixed polynomials, plain loop vs one graph; "
                         "ntt: forward + inverse NTT pairs of --batch columns of 2^--log-n points (--field); "
                         "layout: the Merkle-prep permutations of the BabyBear LDE output")
    ap.add_argument("--lanes", type=int, default=8)
    return ap.parse_args()


def shift_monty(a) -> int:
    """Montgomery form of the coset shift (0 = the reference default)."""
    if a.shift == "reference":
        return 0
    if getattr(a, "field", "bb") == "kb":
        return (3 << 32) % KB_P  # to_monty(3): KoalaBear's multiplicative generator
    return (31 << 32) % BB_P  # to_monty(31) = 31 * 2^32 mod p


def metric_name(a) -> str:
    if a.field == "m31":
        return f"M31 blow-up 2^{a.log_n}x{a.batch} {1 << a.added_bits}x"
    if a.field == "kb":
        return f"KoalaBear coset LDE 2^{a.log_n}x{a.batch} {1 << a.added_bits}x"
    if getattr(a, "natural", False):
        return f"BabyBear coset LDE 2^{a.log_n}x{a.batch} {1 << a.added_bits}x natural-order rows"
    return METRIC if (a.log_n, a.batch, a.added_bits) == (20, 256, 1) else \
        f"BabyBear coset LDE 2^{a.log_n}x{a.batch} {1 << a.added_bits}x"


def workload(a) -> dict:
    if a.field == "m31":
        return {"workload": f"M31 blow-up 2^{a.log_n} x {a.batch} cols, {1 << a.added_bits}x (inverse on odds(log n), "
                            f"zero-pad, forward on odds(log n + added_bits))",
                "log_n": a.log_n, "columns": a.batch, "added_bits": a.added_bits, "layout": "SoA column-major, u32",
                "l2": f"inputs larger than L2 ({4 * a.batch << a.log_n >> 20} MiB in, "
                      f"{4 * a.batch << (a.log_n + a.added_bits) >> 20} MiB out per step)"}
    fname, g = ("KoalaBear", 3) if a.field == "kb" else ("BabyBear", 31)
    return {"workload": f"{fname} coset LDE 2^{a.log_n} x {a.batch} cols, {1 << a.added_bits}x blow-up",
            "log_n": a.log_n, "columns": a.batch, "added_bits": a.added_bits, "mode": a.mode,
            "shift": f"g = {g}, row i times {g}^i" if a.shift == "31" else
                     "two_adic_generator(log_n_ext+1) (reference default)",
            "layout": "SoA column-major, Montgomery u32" +
                      (", natural-order input and output rows" if getattr(a, "natural", False) else
                       ", bit-reversed input and output rows (the reference's convention)"),
            "l2": f"inputs larger than L2 ({4 * a.batch << a.log_n >> 20} MiB in, "
                  f"{4 * a.batch << (a.log_n + a.added_bits) >> 20} MiB out per step)"}


def algorithmic_bytes(a) -> int:
    return 4 * a.batch * (1 << a.log_n) * (1 + (1 << a.added_bits))


# ----------------------------------------------------------------- clocks ---
class ClockSampler:
    """nvidia-smi samples (SM clock, throttle reasons) during the timed region."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.proc = None
        self.lines: list[str] = []
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self, t0: float, t1: float) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [l for (ts, l) in self.lines if t0 - 0.05 <= ts <= t1 + 0.1]
        if not rows:
            rows = [l for (_, l) in self.lines]
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            parts = [p.strip() for p in r.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "of measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "of fallback (6.65 TB/s copy measured earlier on this GPU type; MEASURED_PEAKS.json absent)"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    p = ROOT / "profiles" / "ncu_traffic.txt"
    if p.exists():
        for line in p.read_text().splitlines():
            parts = line.split()
            if len(parts) == 2 and not line.startswith("#") and parts[0] == kernel:
                return int(parts[1])
    return None


# ------------------------------------------------------------ CPU legs ---
def field_p(a) -> int:
    return {"bb": BB_P, "kb": KB_P}.get(a.field, 2147483647)


def dtype_of(a) -> str:
    return {"bb": "u32 (BabyBear Montgomery)", "kb": "u32 (KoalaBear Montgomery)"}.get(a.field, "u32 (M31 canonical)")


def oracle_lde(a, O):
    """The oracle's LDE of the bench's field: f(x, columns, threads)."""
    if a.field == "m31":
        return lambda x, cols, threads: O.m31_lde(x, a.log_n, cols, a.added_bits, threads=threads)
    if a.field == "kb":
        return lambda x, cols, threads: O.kb_coset_lde(x, a.log_n, cols, a.added_bits, shift_monty=shift_monty(a),
                                                       threads=threads)
    return lambda x, cols, threads: O.bb_coset_lde(x, a.log_n, cols, a.added_bits, shift_monty=shift_monty(a),
                                                   threads=threads)


def cpu_lde_sample(a, target_s: float) -> dict:
    """The oracle (reference CPU path restated in C) on a bounded column
    sample, all host threads; returns ms scaled to the full column count."""
    from oracle import oracle as O
    threads = O.default_threads()
    n = 1 << a.log_n
    lde = oracle_lde(a, O)
    one = O.lcg(n, 1, field_p(a), monty=a.field != "m31")
    t = time.perf_counter()
    lde(one, 1, 1)
    t1 = time.perf_counter() - t
    cols = int(max(1, min(a.batch, round(target_s * threads / max(t1, 1e-6)))))
    cols = max(1, min(a.batch, (cols // threads) * threads or cols))
    x = O.lcg(cols << a.log_n, 42 + a.log_n, field_p(a), monty=a.field != "m31")
    t = time.perf_counter()
    lde(x, cols, threads)
    ts = time.perf_counter() - t
    return {"value": ts * 1e3 * a.batch / cols, "unit": "ms", "cores": threads, "kind": "port",
            "sample": f"{cols} of {a.batch} columns (oracle/oracle.c LDE, OpenMP over columns), "
                      f"scaled x{a.batch / cols:.2f}; 1-thread column time {t1 * 1e3:.1f} ms" +
                      ("; the reference-order LDE (natural rows add two permutations)" if getattr(a, "natural", False)
                       else ""),
            "single_thread_ms_full": t1 * 1e3 * a.batch}


def run_reference(a, rank: int) -> None:
    if rank != 0:
        return
    from oracle import oracle as O
    threads = O.default_threads()
    n = 1 << a.log_n
    per_step = max(0.3, min(20.0, 150.0 / max(1, a.steps + a.warmup)))  # whole run ~2.5 min
    lde = oracle_lde(a, O)
    t = time.perf_counter()
    lde(O.lcg(n, 1, field_p(a), monty=a.field != "m31"), 1, 1)
    t1 = time.perf_counter() - t
    cols = int(max(1, min(a.batch, round(per_step * threads / max(t1, 1e-6)))))
    x = O.lcg(cols << a.log_n, 42 + a.log_n, field_p(a), monty=a.field != "m31")
    times = []
    for i in range(a.warmup + a.steps):
        t = time.perf_counter()
        lde(x, cols, threads)
        if i >= a.warmup:
            times.append((time.perf_counter() - t) * a.batch / cols)
    ms = statistics.mean(times) * 1e3
    sample = f"{cols} of {a.batch} columns per step (oracle/oracle.c, OpenMP over columns), scaled x{a.batch / cols:.2f}"
    line = {"impl": "reference", "metric": metric_name(a), "value": ms, "unit": "ms", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": ms / PUBLISHED_MS if metric_name(a) == METRIC else None,
            "dtype": dtype_of(a), "data": "synthetic",
            "config": {**workload(a), "parallelism": f"replicas x{a.gpus}" if a.gpus > 1 else "single GPU"},
            "step_stats": step_stats([t * 1e3 for t in times]),
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU leg ---
def main() -> None:
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank)
        return
    if a.workload in ("uneven", "served", "table", "ntt", "layout"):
        if rank == 0:  # single-GPU workloads: under torchrun the other ranks have no work
            {"uneven": run_uneven, "served": run_served, "table": run_table, "ntt": run_ntt,
             "layout": run_layout}[a.workload](a)
        return

    import torch
    import sfntt
    from sfntt.replicas import Replicas, job_time_per_unit

    torch.cuda.set_device(local)
    # N GPUs = N independent replicas; the process group only carries the
    # barrier and the max of per-rank times (no data-path collective)
    rep = Replicas(backend="nccl", timeout_s=120, device=torch.device("cuda", local))
    barrier, max_all = rep.barrier, rep.max

    ctx = sfntt.Context(local)
    m31 = a.field == "m31"
    n, n_ext = 1 << a.log_n, 1 << (a.log_n + a.added_bits)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234 + rank)
    x = torch.randint(0, field_p(a), (a.batch * n,), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    out = torch.empty(a.batch * n_ext, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    shift = shift_monty(a)
    if m31:
        lde = sfntt.M31Lde(ctx)
        ctx.prepare_lde(sfntt.FIELD_M31, a.log_n, a.added_bits)

        def step():
            lde.execute_dev(x.data_ptr(), out.data_ptr(), a.log_n, a.batch, a.added_bits, stream=stream)

        def host_call(hin, hout):
            lde.execute(hin, a.log_n, a.batch, a.added_bits, out=hout)
    else:
        fid = sfntt.FIELD_KOALABEAR if a.field == "kb" else sfntt.FIELD_BABYBEAR
        lde = (sfntt.KbCosetLdeBatch if a.field == "kb" else sfntt.CosetLdeBatch)(ctx, fused=(a.mode == "fused"),
                                                                               natural=a.natural)
        sfntt.convert_monty_dev(ctx, fid, x.data_ptr(), x.numel(), to_monty=True, stream=stream)
        ctx.prepare_lde(fid, a.log_n, a.added_bits, shift)

        def step():
            lde.execute_dev(x.data_ptr(), out.data_ptr(), a.log_n, a.batch, a.added_bits, shift_monty=shift,
                            stream=stream)

        def host_call(hin, hout):
            lde.execute(hin, a.log_n, a.batch, a.added_bits, shift_monty=shift, out=hout)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()

    gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    sampler = ClockSampler(gpu_id)
    time.sleep(0.6)
    launches0 = ctx.launch_count()
    barrier()
    torch.cuda.synchronize()
    # one event per step boundary on the launching stream: the total and the
    # per-step spread come from the same timed run
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    w0 = time.time()
    evs[0].record()
    for i in range(a.steps):
        step()
        evs[i + 1].record()
    torch.cuda.synchronize()
    w1 = time.time()
    barrier()
    ev0, ev1 = evs[0], evs[-1]
    per_step = [evs[i].elapsed_time(evs[i + 1]) for i in range(a.steps)]
    launches = ctx.launch_count() - launches0
    clocks = sampler.stop(w0, w1)
    # per-kernel breakdown on a separate run: events around every launch
    # would stop consecutive passes from overlapping their launch gaps
    ctx.kernel_timing(True)
    for _ in range(min(20, a.steps)):
        step()
    torch.cuda.synchronize()
    kt = ctx.kernel_times()
    ctx.kernel_timing(False)
    step_ms = max_all(ev0.elapsed_time(ev1) / a.steps)
    value = job_time_per_unit(step_ms, world)

    # dominant kernel and its roofline
    peak, peak_kind = peaks()
    dom = max(kt.items(), key=lambda kv: kv[1][1])
    name, (nl, tot_ms, nbytes) = dom
    avg_ms = tot_ms / nl
    achieved = (nbytes / nl) / (avg_ms * 1e-3) / 1e9
    traffic = ncu_traffic(name)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": name, "kernel_ms": avg_ms,
                "algorithmic_bytes_per_launch": nbytes // nl, "peak_kind": peak_kind}
    kernels = {k: {"launches": v[0], "avg_ms": v[1] / v[0], "share": v[1] / sum(t[1] for t in kt.values()),
                   "gbs": (v[2] / v[0]) / (v[1] / v[0] * 1e-3) / 1e9} for k, v in kt.items()}
    lde_gbs = algorithmic_bytes(a) / (step_ms * 1e-3) / 1e9
    # integer roofline: radix-2 butterflies of the LDE (the zero-padded top
    # added_bits layers are multiplications only) against the measured
    # register-resident butterfly rate of this GPU
    bf_peak = {"gs": ctx.butterfly_peak(True), "ct": ctx.butterfly_peak(False)}
    lde_bf = a.batch * ((n // 2) * a.log_n + (n_ext // 2) * a.log_n)
    dom_bf = kernel_butterflies(name, nbytes // nl, a.added_bits)
    int_roofline = {"bound": "int32 issue", "unit": "butterflies/s",
                    "peak": bf_peak["gs"], "peak_ct": bf_peak["ct"],
                    "peak_kind": "measured on this GPU (sfntt_butterfly_peak, register-resident butterflies)",
                    "lde_achieved": lde_bf / (step_ms * 1e-3), "lde_frac": lde_bf / (step_ms * 1e-3) / bf_peak["gs"],
                    "kernel": name, "kernel_achieved": dom_bf / (avg_ms * 1e-3),
                    "kernel_frac": dom_bf / (avg_ms * 1e-3) / bf_peak["gs"]}

    # end to end through the host-buffer C-ABI call (copies inside the timed region)
    e2e = None
    if not a.no_e2e:
        hin = ctx.pinned(a.batch * n)
        hout = ctx.pinned(a.batch * n_ext)
        hin.array[:] = x.cpu().numpy().view("uint32")
        host_call(hin.array, hout.array)  # warm-up
        barrier()
        ts = []
        for _ in range(a.e2e_steps):
            t = time.perf_counter()
            host_call(hin.array, hout.array)
            ts.append(time.perf_counter() - t)
        e2e_ms = max_all(statistics.mean(ts) * 1e3)
        ok = bool((hout.array[: n_ext] == out[: n_ext].cpu().numpy().view("uint32")).all())
        e2e = {"value": e2e_ms / world, "unit": "ms", "h2d_bytes_per_step": 4 * a.batch * n,
               "d2h_bytes_per_step": 4 * a.batch * n_ext, "steps": a.e2e_steps,
               "path": ("sfntt_m31_lde" if m31 else "sfntt_bb_coset_lde") +
                       " (pinned host buffers, column chunks pipelined over 3 streams)",
               "matches_device_run": ok}
        hin.free()
        hout.free()

    secondary = None if a.no_secondary else secondary_metrics(ctx, sfntt, torch)
    layouts = None if (a.no_secondary or m31) else layout_metrics(a, ctx, sfntt, torch, x, out, stream)
    del x, out
    torch.cuda.empty_cache()
    served = None if (a.no_served or world > 1) else served_sweep(a, ctx, sfntt, torch)
    uneven = None if (a.no_uneven or world > 1 or m31) else uneven_metrics(a, ctx, sfntt, torch)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_lde_sample(a, a.cpu_seconds)

    rep.close()
    if rank != 0:
        return
    line = {"metric": metric_name(a), "value": value, "unit": "ms", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": step_ms, "higher_is_better": False, "scaling": "weak",
            "step_stats": step_stats(per_step),
            "vs_baseline": value / PUBLISHED_MS if metric_name(a) == METRIC else None,
            "dtype": dtype_of(a)[:-1] + ", exact)",
            "data": "synthetic: seeded uniform canonical values in [0, p)" + ("" if m31 else ", Montgomery on device"),
            "config": {**workload(a), "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "gpu_launches": launches, "launches_per_step": launches / a.steps,
            "lde_gbs": lde_gbs, "lde_hbm_frac": lde_gbs / peak,
            "melem_per_s_out": a.batch * n_ext / (value * 1e-3) / 1e6,
            "roofline": roofline, "int_roofline": int_roofline, "kernels": kernels, "clocks": clocks, "e2e": e2e,
            "cpu_baseline": cpu,
            "secondary": secondary, "layout": layouts, "served": served, "device": ctx.device_info()}
    line.update(headline_keys(secondary, uneven, served))
    if uneven is not None:
        line["uneven"] = uneven
    print(json.dumps(line), flush=True)


def step_stats(ms: list) -> dict:
    """Spread of the per-step device times (the reference's bench reports
    median, min, max, stddev, p95 and CV: benches/ntt_benchmark.rs:63-120)."""
    import numpy as np
    v = np.asarray(ms, dtype=float)
    mean = float(v.mean())
    sd = float(v.std(ddof=1)) if v.size > 1 else 0.0
    return {"mean_ms": mean, "median_ms": float(np.median(v)), "min_ms": float(v.min()), "max_ms": float(v.max()),
            "p95_ms": float(np.percentile(v, 95)), "stddev_ms": sd, "cv_pct": 100.0 * sd / mean if mean else 0.0,
            "n": int(v.size)}


def headline_keys(secondary, uneven, served) -> dict:
    """The other configurations' headline numbers as top-level scalars:
    the M31 2^16 forward + inverse pair, the BabyBear 2^10..2^24 pairs, the
    uneven batch (plain loop and one launch) and the served stream at its
    highest rate."""
    out = {}
    if secondary:
        out["m31_2^16_fwd_inv_us"] = secondary["m31"]["16"]["fwd_inv_us"]
        for k in ("10", "16", "20", "21", "22", "24"):
            out[f"bb_2^{k}_fwd_inv_us"] = secondary["bb"][k]["fwd_inv_us"]
        out["bb_2^24_gelem_s"] = secondary["bb"]["24"]["gelem_s"]
    if uneven:
        for k in ("plain_loop_ms", "graph_ms", "persistent_ms", "speedup", "persistent_speedup", "persistent_vs_graph"):
            if k in uneven:
                out[f"uneven_{k}"] = uneven[k]
    if served:
        for prefix, top in (("served", served["at_max_rate"]), ("served_small", served["small"]["at_max_rate"])):
            out[f"{prefix}_rate_req_s"] = top["rate"]
            out[f"{prefix}_melem_s"] = top["served_melem_s"]
            out[f"{prefix}_plain_melem_s"] = top["plain_melem_s"]
            out[f"{prefix}_throughput_ratio"] = top["throughput_ratio"]
            out[f"{prefix}_p99_ms"] = top["served_p99_ms"]
            out[f"{prefix}_plain_p99_ms"] = top["plain_p99_ms"]
    return out


def layout_metrics(a, ctx, sfntt, torch, x, out, stream) -> dict:
    """The callers either side of the LDE: natural row order (Plonky3's
    coset_lde_batch convention) and the row-major Merkle-commitment layout of
    the LDE output (HBM-bound permutations: every word read and written once),
    plus the whole LDE in the natural-order convention."""
    n_ext = 1 << (a.log_n + a.added_bits)
    total = a.batch * n_ext
    peak, _ = peaks()
    rows = torch.empty_like(out)

    def timed(fn, reps=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    res = {"workload": f"LDE output, {a.batch} columns x 2^{a.log_n + a.added_bits} rows ({4 * total / 2**30:.0f} GiB)"}
    lb = a.log_n + a.added_bits
    for name, fn in (("natural_in_place", lambda: sfntt.layout_dev(ctx, out.data_ptr(), out.data_ptr(), lb, a.batch,
                                                                   sfntt.LAYOUT_NATURAL, stream)),
                     ("row_major", lambda: sfntt.layout_dev(ctx, out.data_ptr(), rows.data_ptr(), lb, a.batch,
                                                            sfntt.LAYOUT_ROW_MAJOR, stream)),
                     ("row_major_natural", lambda: sfntt.layout_dev(ctx, out.data_ptr(), rows.data_ptr(), lb, a.batch,
                                                                    sfntt.LAYOUT_ROW_MAJOR | sfntt.LAYOUT_NATURAL,
                                                                    stream))):
        ms = timed(fn)
        gbs = 8 * total / (ms * 1e-3) / 1e9
        res[name] = {"ms": ms, "gbs": gbs, "hbm_frac": gbs / peak}
    lde_nat = sfntt.CosetLdeBatch(ctx, natural=True)
    ms = timed(lambda: lde_nat.execute_dev(x.data_ptr(), out.data_ptr(), a.log_n, a.batch, a.added_bits, stream=stream))
    res["lde_natural_order_ms"] = ms
    # the M31 blow-up of the same shape (inputs < BabyBear p are canonical M31 values)
    m31 = sfntt.M31Lde(ctx)
    ctx.prepare_lde(sfntt.FIELD_M31, a.log_n, a.added_bits)
    res["m31_lde_ms"] = timed(lambda: m31.execute_dev(x.data_ptr(), out.data_ptr(), a.log_n, a.batch, a.added_bits,
                                                      stream=stream))
    # the canonic-coset circle LDE of the same shape (M31 network, circle-FFT twiddles)
    circ = sfntt.CircleLde(ctx)
    circ.prepare(a.log_n, a.added_bits)
    res["circle_lde_ms"] = timed(lambda: circ.execute_dev(x.data_ptr(), out.data_ptr(), a.log_n, a.batch,
                                                          a.added_bits, stream=stream))
    # the KoalaBear coset LDE of the same shape (words < BabyBear p are valid KoalaBear Montgomery words)
    kb = sfntt.KbCosetLdeBatch(ctx)
    ctx.prepare_lde(sfntt.FIELD_KOALABEAR, a.log_n, a.added_bits)
    res["kb_lde_ms"] = timed(lambda: kb.execute_dev(x.data_ptr(), out.data_ptr(), a.log_n, a.batch, a.added_bits,
                                                    stream=stream))
    del rows
    return res


SMALL_STREAM = {"log_n_weights": {14: 1, 15: 1, 16: 1}, "cols_range": (8, 32),
                "rates": (1000.0, 5000.0, 20000.0, 100000.0, 1000000.0)}


def _trace_stats(lat, mk, elems_out, bytes_alg, peak, launches=None) -> dict:
    import numpy as np
    d = {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
         "mean_ms": float(lat.mean() * 1e3), "makespan_s": mk,
         "melem_per_s": elems_out / mk / 1e6, "hbm_frac": bytes_alg / mk / (peak * 1e9)}
    if launches is not None:
        d["launches"] = launches
    return d


def _replay_stream(a, ctx, sfntt, reqs, unit_arrivals, rates, budget, peak, host=None, dropin=None) -> list:
    """One stream at each rate: the plain sequential per-request loop (one
    slot, one launch per request), continuous batching (--slots slots, one
    launch per request) and continuous batching with packing (up to --pack
    same-shape requests per launch); `dropin` (optional) replays the
    drop-in per-request host call."""
    elems_out = sum(it["batch"] << (it["log_n"] + it["added_bits"]) for it in reqs)
    bytes_alg = sum(4 * (it["batch"] << it["log_n"]) * (1 + (1 << it["added_bits"])) for it in reqs)
    out = []
    for rate in rates:
        arr = unit_arrivals / rate
        row = {"rate_req_s": rate}
        for name, slots, pack in (("plain", 1, 1), ("served", a.slots, 1), ("packed", a.slots, a.pack)):
            st = {}
            lat, mk = sfntt.serve_trace(ctx, reqs, arr, slots=slots, budget_bytes=budget, host=host, max_pack=pack,
                                        stats=st)
            row[name] = _trace_stats(lat, mk, elems_out, bytes_alg, peak, st.get("launches"))
        if dropin is not None:
            lat, mk = dropin(arr)
            row["dropin_host_call"] = _trace_stats(lat, mk, elems_out, bytes_alg, peak, len(reqs))
        for name in ("served", "packed"):
            row[f"{name}_throughput_ratio"] = row[name]["melem_per_s"] / row["plain"]["melem_per_s"]
            row[f"{name}_p99_ratio"] = row[name]["p99_ms"] / row["plain"]["p99_ms"]
        row["throughput_ratio"] = row["packed_throughput_ratio"]
        row["p99_ratio"] = row["packed_p99_ratio"]
        out.append(row)
    return out


def served_sweep(a, ctx, sfntt, torch) -> dict:
    """The served streams, each replayed at several Poisson arrival rates
    through the plain sequential per-request loop, continuous batching and
    continuous batching with packing (same arena, kernels and resident tables):
      mixed -- the configured stream: field 50/50 M31 / BabyBear, log n 14..22
               weighted toward 18-20, 8..256 columns, blow-up 2 or 4, seeded;
               inputs are seeded slices of one resident 4 GiB pool;
      small -- requests that leave most of the GPU idle (log n 14..16, 8..32
               columns), inputs resident on the device; then the same
               requests from host memory (input copied in, output copied
               back) at the highest rate, beside the drop-in per-request host
               call replayed in order.
    HBM admission budget --budget-gb; latency = completion seen by the host -
    arrival."""
    import numpy as np
    rates = [float(r) for r in a.rates.split(",") if r]
    budget = int(a.budget_gb * (1 << 30))
    peak, _ = peaks()
    pool_words = 1 << 30
    gen = torch.Generator(device="cuda")
    gen.manual_seed(4242)
    pool = torch.randint(0, BB_P, (pool_words,), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    reqs, unit_arrivals = sfntt.served_workload(a.requests, rate=1.0, seed=2025)
    rng = np.random.default_rng(77)
    for it in reqs:
        need = it["batch"] << it["log_n"]
        off = int(rng.integers(0, (pool_words - need) // 64 + 1)) * 64
        it["d_in"] = pool.data_ptr() + 4 * off
    # warm-up: tables, the arena and every kernel shape once
    sfntt.serve_trace(ctx, reqs, np.zeros(len(reqs)), slots=a.slots, budget_bytes=budget, max_pack=a.pack)
    launches0 = ctx.launch_count()
    mixed = _replay_stream(a, ctx, sfntt, reqs, unit_arrivals, rates, budget, peak)
    launches = ctx.launch_count() - launches0
    del pool
    torch.cuda.empty_cache()

    # the small-request stream: device inputs (slices of a resident pool) at
    # each rate, then host requests at the highest rate beside the drop-in call
    sreqs, s_unit = sfntt.served_workload(a.requests, rate=1.0, seed=2026,
                                          cols_range=SMALL_STREAM["cols_range"],
                                          log_n_weights=SMALL_STREAM["log_n_weights"])
    spool_words = 1 << 26
    spool = torch.randint(0, BB_P, (spool_words,), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    for it in sreqs:
        need = it["batch"] << it["log_n"]
        off = int(rng.integers(0, (spool_words - need) // 64 + 1)) * 64
        it["d_in"] = spool.data_ptr() + 4 * off
    sfntt.serve_trace(ctx, sreqs, np.zeros(len(sreqs)), slots=a.slots, budget_bytes=budget, max_pack=a.pack)
    small = _replay_stream(a, ctx, sfntt, sreqs, s_unit, SMALL_STREAM["rates"], budget, peak)
    del spool
    host = []
    for i, it in enumerate(sreqs):
        p = BB_P if it["field"] == sfntt.FIELD_BABYBEAR else 2147483647
        x = ctx.pinned(it["batch"] << it["log_n"])
        x.array[:] = np.random.default_rng(500 + i).integers(0, p, x.array.size, dtype=np.uint32)
        if it["field"] == sfntt.FIELD_BABYBEAR:
            x.array[:] = ((x.array.astype(np.uint64) << 32) % BB_P).astype(np.uint32)  # Montgomery form
        y = ctx.pinned(it["batch"] << (it["log_n"] + it["added_bits"]))
        host.append((x, y))
    host_arrays = [(x.array, y.array) for x, y in host]
    ldes = {sfntt.FIELD_BABYBEAR: sfntt.CosetLdeBatch(ctx), sfntt.FIELD_M31: sfntt.M31Lde(ctx)}

    def dropin(arr):
        """The drop-in call per request (sfntt_coset_lde / sfntt_m31_lde, host
        buffers, synchronous), one after another as they arrive."""
        lat = np.zeros(len(sreqs))
        t0 = time.perf_counter()
        for i, it in enumerate(sreqs):
            while time.perf_counter() - t0 < arr[i]:
                pass
            ldes[it["field"]].execute(host_arrays[i][0], it["log_n"], it["batch"], it["added_bits"],
                                      out=host_arrays[i][1])
            lat[i] = time.perf_counter() - t0 - arr[i]
        return lat, time.perf_counter() - t0

    dropin(np.zeros(len(sreqs)))  # warm-up: tables and staging buffers
    sfntt.serve_trace(ctx, sreqs, np.zeros(len(sreqs)), slots=a.slots, budget_bytes=budget, host=host_arrays,
                      max_pack=a.pack)
    small_host = _replay_stream(a, ctx, sfntt, sreqs, s_unit, SMALL_STREAM["rates"][-1:], budget, peak,
                                host=host_arrays, dropin=dropin)
    for x, y in host:
        x.free()
        y.free()

    def summary(rows):
        top = max(rows, key=lambda r: r["rate_req_s"])
        return {"rate": top["rate_req_s"], "plain_p50_ms": top["plain"]["p50_ms"],
                "plain_p99_ms": top["plain"]["p99_ms"], "served_p50_ms": top["packed"]["p50_ms"],
                "served_p99_ms": top["packed"]["p99_ms"], "plain_melem_s": top["plain"]["melem_per_s"],
                "served_melem_s": top["packed"]["melem_per_s"], "throughput_ratio": top["packed_throughput_ratio"],
                "unpacked_throughput_ratio": top["served_throughput_ratio"]}

    return {"workload": f"{a.requests} requests per rate, Poisson arrivals, field 50/50, log n 14..22 weighted "
                        f"18-20, columns U[8,256], blow-up 2/4, seed 2025; inputs: slices of a resident 4 GiB pool",
            "slots": a.slots, "max_pack": a.pack, "budget_gb": a.budget_gb, "requests": a.requests,
            "gpu_launches": launches,
            "at_max_rate": summary(mixed), "sweep": mixed,
            "small": {"workload": f"{a.requests} requests per rate, field 50/50, log n 14..16, columns U[8,32], "
                                  "blow-up 2/4, seed 2026; inputs: slices of a resident 256 MiB pool",
                      "at_max_rate": summary(small), "sweep": small,
                      "host_requests": {"note": "the same requests from pinned host memory (input copied in, output "
                                                "copied back: bound by the PCIe copies), and the drop-in host call "
                                                "per request",
                                        "sweep": small_host}}}


def run_served(a) -> None:
    import torch
    import sfntt
    torch.cuda.set_device(0)
    ctx = sfntt.Context(0)
    res = served_sweep(a, ctx, sfntt, torch)
    top = res["at_max_rate"]
    line = {"metric": "served stream p50/p99 and Melem/s vs plain loop", "unit": "Melem/s",
            "value": top["served_melem_s"], "higher_is_better": True, "plain_loop_melem_s": top["plain_melem_s"],
            "served": res, "data": "synthetic", "device": ctx.device_info()}
    print(json.dumps(line), flush=True)


def run_ntt(a) -> None:
    """Forward + inverse NTT pairs (the single-column configurations: M31
    2^16, BabyBear 2^10..2^24) on device-resident columns: 10 pairs captured
    in a CUDA graph, replayed --steps times after --warmup plain pairs; then
    the per-kernel device times of 10 more pairs."""
    import torch
    import sfntt
    torch.cuda.set_device(0)
    ctx = sfntt.Context(0)
    field = {"bb": sfntt.FIELD_BABYBEAR, "m31": sfntt.FIELD_M31, "kb": sfntt.FIELD_KOALABEAR}[a.field]
    backend = {"bb": sfntt.BbCudaCtGsR4, "m31": sfntt.CudaCtGsR4, "kb": sfntt.KbCudaCtGsR4}[a.field](ctx)
    p = {"bb": BB_P, "m31": 2147483647, "kb": KB_P}[a.field]
    log_n, cols = a.log_n, a.batch
    gen = torch.Generator(device="cuda")
    gen.manual_seed(2024)
    d = torch.randint(0, p, (cols << log_n,), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    ptr = d.data_ptr()
    ctx.prepare(field, log_n)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(max(a.warmup, 3)):
        backend.forward_dev(ptr, log_n, cols, stream)
        backend.inverse_dev(ptr, log_n, cols, stream)
    torch.cuda.synchronize()
    graph, per_graph = torch.cuda.CUDAGraph(), 10
    with torch.cuda.graph(graph):
        cs = torch.cuda.current_stream().cuda_stream
        for _ in range(per_graph):
            backend.forward_dev(ptr, log_n, cols, cs)
            backend.inverse_dev(ptr, log_n, cols, cs)
    graph.replay()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    del graph
    us = e0.elapsed_time(e1) * 1e3 / (a.steps * per_graph)
    ctx.kernel_timing(True)
    for _ in range(per_graph):
        backend.forward_dev(ptr, log_n, cols, stream)
        backend.inverse_dev(ptr, log_n, cols, stream)
    torch.cuda.synchronize()
    kt = ctx.kernel_times()
    ctx.kernel_timing(False)
    elems = cols << log_n
    peak, peak_kind = peaks()
    line = {"metric": f"{a.field} NTT forward+inverse 2^{log_n} x {cols}", "value": us, "unit": "us",
            "higher_is_better": False, "steps": a.steps, "warmup": a.warmup,
            "gelem_s": 2 * elems / (us * 1e-6) / 1e9,
            "hbm_frac": 16 * elems / (us * 1e-6) / 1e9 / peak, "peak_kind": peak_kind,
            "kernels": {k: {"launches": v[0], "avg_us": 1e3 * v[1] / v[0]} for k, v in kt.items()},
            "data": "synthetic: seeded uniform values in [0, p), device-resident",
            "config": {"workload": f"{a.field} forward + inverse NTT, {cols} column(s) of 2^{log_n} points",
                       "l2": "columns of up to 2^24 words stay resident in L2 (126 MB)"},
            "device": ctx.device_info()}
    print(json.dumps(line), flush=True)


def run_layout(a) -> None:
    """The Merkle-prep permutations of one BabyBear 2x LDE output (--batch
    columns of 2^(--log-n + --added-bits) rows): natural row order in place,
    row-major, row-major in natural order (layout_metrics' first three rows)."""
    import torch
    import sfntt
    torch.cuda.set_device(0)
    ctx = sfntt.Context(0)
    n, n_ext = 1 << a.log_n, 1 << (a.log_n + a.added_bits)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234)
    x = torch.randint(0, BB_P, (a.batch * n,), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    out = torch.empty(a.batch * n_ext, dtype=torch.int32, device="cuda")
    rows = torch.empty_like(out)
    stream = torch.cuda.current_stream().cuda_stream
    sfntt.CosetLdeBatch(ctx).execute_dev(x.data_ptr(), out.data_ptr(), a.log_n, a.batch, a.added_bits, stream=stream)
    lb, total = a.log_n + a.added_bits, a.batch * n_ext
    peak, peak_kind = peaks()
    res = {}
    for name, flags, dst in (("natural_in_place", sfntt.LAYOUT_NATURAL, out),
                             ("row_major", sfntt.LAYOUT_ROW_MAJOR, rows),
                             ("row_major_natural", sfntt.LAYOUT_ROW_MAJOR | sfntt.LAYOUT_NATURAL, rows)):
        fn = lambda: sfntt.layout_dev(ctx, out.data_ptr(), dst.data_ptr(), lb, a.batch, flags, stream)
        for _ in range(max(a.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        res[name] = {"ms": ms, "gbs": 8 * total / (ms * 1e-3) / 1e9, "hbm_frac": 8 * total / (ms * 1e-3) / 1e9 / peak}
    line = {"metric": f"Merkle-prep layouts of the 2^{lb} x {a.batch} LDE output", "unit": "ms",
            "value": res["row_major"]["ms"], "higher_is_better": False, "steps": a.steps, "warmup": a.warmup,
            "layouts": res, "peak_kind": peak_kind, "data": "synthetic",
            "config": {"workload": f"BabyBear 2x LDE output, {a.batch} columns x 2^{lb} rows, permuted on device",
                       "algorithmic_bytes": 8 * total}, "device": ctx.device_info()}
    print(json.dumps(line), flush=True)


def run_uneven(a) -> None:
    import torch
    import sfntt
    torch.cuda.set_device(0)
    print(json.dumps(uneven_metrics(a, sfntt.Context(0), sfntt, torch)), flush=True)


def uneven_metrics(a, ctx, sfntt, torch) -> dict:
    """The uneven-batch configuration: 64 polynomials, field 50/50 M31 /
    BabyBear, log n uniform in 12..22, 1..128 columns, blow-up 1/2/4 with
    probability 1/3 each, seeded; one plain launch sequence per polynomial vs
    one autotuned CUDA-graph launch for the whole batch (per-item kernels on 8
    lanes) vs the persistent form (one work-list launch per LDE phase for every
    2^13..2^20-point item, the rest per item beside it), outputs compared."""
    items = sfntt.uneven_workload(64, seed=2024)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(99)
    keep = []
    stream = torch.cuda.current_stream().cuda_stream
    for it in items:
        p = BB_P if it["field"] == sfntt.FIELD_BABYBEAR else 2147483647
        x = torch.randint(0, p, (it["batch"] << it["log_n"],), dtype=torch.int64, device="cuda",
                          generator=gen).to(torch.int32)
        if it["field"] == sfntt.FIELD_BABYBEAR:
            sfntt._check(ctx.handle, sfntt._ffi.lib().sfntt_bb_to_monty_dev(ctx.handle, x.data_ptr(), x.numel(), stream))
        y = torch.empty(it["batch"] << (it["log_n"] + it["added_bits"]), dtype=torch.int32, device="cuda")
        it["d_in"], it["d_out"] = x.data_ptr(), y.data_ptr()
        keep.append((x, y))
    batch = sfntt.LdeBatch(ctx, items)
    batch.prepare()
    t0 = time.perf_counter()
    batch.autotune(reps=1)
    tune_s = time.perf_counter() - t0
    plans = [batch.plan_of(i) for i in range(len(items))]

    def timed(fn, steps):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def digest():
        return [int(y.view(torch.int64 if y.numel() % 2 == 0 else torch.int32).sum().item()) for _, y in keep]

    steps = max(3, min(a.steps, 20))
    plain_ms = timed(lambda: batch.run(stream), steps)
    d_plain = digest()
    for _, y in keep:
        y.zero_()
    g = batch.graph(lanes=a.lanes)
    graph_ms = timed(lambda: g.launch(stream), steps)
    d_graph = digest()
    # persistent form: the eligible items' three phases as one work-list launch each
    for _, y in keep:
        y.zero_()
    pg = batch.persistent_graph(lanes=a.lanes)
    persistent_ms = timed(lambda: pg.launch(stream), steps)
    d_persistent = digest()
    persistent_kernels = pg.kernel_count()
    pg.close()
    elems_out = sum(it["batch"] << (it["log_n"] + it["added_bits"]) for it in items)
    bytes_alg = sum(4 * (it["batch"] << it["log_n"]) * (1 + (1 << it["added_bits"])) for it in items)
    peak, peak_kind = peaks()
    line = {"metric": "uneven batch: 64 mixed M31/BabyBear LDEs", "unit": "ms", "value": graph_ms,
            "plain_loop_ms": plain_ms, "graph_ms": graph_ms, "speedup": plain_ms / graph_ms,
            "persistent_ms": persistent_ms, "persistent_speedup": plain_ms / persistent_ms,
            "persistent_vs_graph": graph_ms / persistent_ms, "kernels_in_persistent_graph": persistent_kernels,
            "persistent_outputs_identical": d_plain == d_persistent,
            "higher_is_better": False, "steps": steps, "warmup": a.warmup, "lanes": a.lanes,
            "kernels_in_graph": g.kernel_count(), "outputs_identical": d_plain == d_graph,
            "melem_per_s_out": elems_out / (graph_ms * 1e-3) / 1e6,
            "hbm_frac": bytes_alg / (graph_ms * 1e-3) / (peak * 1e9), "autotune_s": tune_s,
            "plans": {str(p): plans.count(p) for p in sorted(set(plans))},
            "config": {"workload": "64 polynomials, field 50/50, log n U[12,22], columns U[1,128], "
                                   "blow-up 1/2/4 (p = 1/3 each), seed 2024", "output_gb": bytes_alg / 1e9},
            "data": "synthetic", "device": ctx.device_info()}
    g.close()
    del keep
    torch.cuda.empty_cache()
    return line


def run_table(a) -> None:
    """Every row of the measurement table, GPU beside the oracle on this host's
    cores (the CPU legs run the oracle, oracle/oracle.c, as the reference's CPU
    path restated; medians of up to 20 runs after up to 5 warm-ups within a
    time bound per row):
      C1  M31 forward + inverse, n = 2^16, one column
      C2  BabyBear forward + inverse, log n 10..24, one column (a single column
          does not split across cores, so the CPU leg is one thread)
      C3  BabyBear coset LDE 2^20 x 256, 2x and 4x, fused and unfused (CPU: one
          column on one thread scaled to 256; all cores on a column sample)
      C4  uneven batch: plain per-polynomial loop vs one graph launch (CPU: one
          column of every polynomial on one thread, scaled by its columns)
      C5  served stream vs the plain loop (see served_sweep)."""
    import copy
    import torch
    import sfntt
    from oracle import oracle as O
    torch.cuda.set_device(0)
    ctx = sfntt.Context(0)
    threads = O.default_threads()
    peak, _ = peaks()

    def cpu_median_ms(fn, budget_s=3.0):
        t = time.perf_counter()
        fn()
        first = time.perf_counter() - t
        reps = int(max(1, min(20, budget_s / max(first, 1e-6))))
        for _ in range(min(5, reps // 4)):
            fn()
        ts = []
        for _ in range(reps):
            t = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t)
        return statistics.median(ts) * 1e3

    res = {"cores": threads}
    sweep = secondary_metrics(ctx, sfntt, torch)
    x16 = O.lcg(1 << 16, 12345 + (1 << 16), O.M31_P)
    res["C1"] = {"gpu_us": sweep["m31"]["16"]["fwd_inv_us"],
                 "cpu_1t_us": cpu_median_ms(lambda: O.m31_inverse(O.m31_forward(x16))) * 1e3,
                 "gpu_hbm_frac": sweep["m31"]["16"]["hbm_frac"], "note": "L2-resident"}
    c2 = {}
    for log_n in range(10, 25):
        x = O.lcg(1 << log_n, 7 + log_n, O.BB_P, monty=True)
        g = sweep["bb"][str(log_n)]
        c2[str(log_n)] = {"gpu_us": g["fwd_inv_us"], "gpu_gelem_s": g["gelem_s"], "gpu_hbm_frac": g["hbm_frac"],
                          "cpu_1t_us": cpu_median_ms(lambda: O.bb_inverse(O.bb_forward(x)), 2.0) * 1e3}
    res["C2"] = c2
    # C3
    n = 1 << 20
    xin = torch.randint(0, BB_P, (256 * n,), dtype=torch.int64, device="cuda").to(torch.int32)
    stream = torch.cuda.current_stream().cuda_stream
    c3 = {}
    for added in (1, 2):
        out = torch.empty(256 * (n << added), dtype=torch.int32, device="cuda")
        row = {}
        for fused in (True, False):
            lde = sfntt.CosetLdeBatch(ctx, fused=fused)
            ctx.prepare_lde(sfntt.FIELD_BABYBEAR, 20, added, shift_monty(a))
            f = lambda: lde.execute_dev(xin.data_ptr(), out.data_ptr(), 20, 256, added,
                                        shift_monty=shift_monty(a), stream=stream)
            for _ in range(3):
                f()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(10):
                f()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 10
            row["gpu_fused_ms" if fused else "gpu_unfused_ms"] = ms
        row["gpu_hbm_frac"] = 4 * 256 * n * (1 + (1 << added)) / (row["gpu_fused_ms"] * 1e-3) / (peak * 1e9)
        b = copy.copy(a)
        b.log_n, b.batch, b.added_bits = 20, 256, added
        cpu = cpu_lde_sample(b, 12.0)
        row["cpu_all_cores_ms"] = cpu["value"]
        row["cpu_1t_ms"] = cpu["single_thread_ms_full"]
        c3[f"{1 << added}x"] = row
        del out
        torch.cuda.empty_cache()
    res["C3"] = c3
    del xin
    torch.cuda.empty_cache()
    # C4
    un = uneven_metrics(a, ctx, sfntt, torch)
    items = sfntt.uneven_workload(64, seed=2024)
    cpu_1t = 0.0
    for k, it in enumerate(items):
        bb = it["field"] == sfntt.FIELD_BABYBEAR
        col = O.lcg(1 << it["log_n"], 500 + k, O.BB_P if bb else O.M31_P, monty=bb)
        t = time.perf_counter()
        if bb:
            O.bb_coset_lde(col, it["log_n"], 1, it["added_bits"], threads=1)
        else:
            O.m31_lde(col, it["log_n"], 1, it["added_bits"], threads=1)
        cpu_1t += (time.perf_counter() - t) * it["batch"]
    res["C4"] = {"gpu_plain_ms": un["plain_loop_ms"], "gpu_graph_ms": un["graph_ms"],
                 "gpu_persistent_ms": un["persistent_ms"], "gpu_hbm_frac": un["hbm_frac"],
                 "outputs_identical": un["outputs_identical"] and un["persistent_outputs_identical"],
                 "cpu_1t_ms": cpu_1t * 1e3}
    # C5
    sv = served_sweep(a, ctx, sfntt, torch)
    def rows(sweep):
        return [{"rate": r["rate_req_s"], **{f"{m}_{k}": r[m][k] for m in ("plain", "served", "packed")
                                              for k in ("p50_ms", "p99_ms", "melem_per_s")},
                 "packed_hbm_frac": r["packed"]["hbm_frac"]} for r in sweep]
    res["C5"] = {"at_max_rate": sv["at_max_rate"], "sweep": rows(sv["sweep"]),
                 "small": {"at_max_rate": sv["small"]["at_max_rate"], "sweep": rows(sv["small"]["sweep"])}}
    print(json.dumps({"metric": "measurement table (C1-C5)", "rows": res, "device": ctx.device_info()}), flush=True)


def kernel_butterflies(name: str, bytes_per_launch: int, added_bits: int) -> float:
    """Radix-2 butterflies of one launch, from its label and algorithmic bytes
    (pass kernels move each point once each way; the expand reads a tile and
    writes 2^added_bits blocks, running P layers on the input and on every block)."""
    import re
    m = re.search(r"_([CS])(\d+)", name)
    layers = int(m.group(2)) if m else 1
    if "expand" in name:
        elems_in = bytes_per_launch / (4 * (1 + (1 << added_bits)))
        return elems_in / 2 * layers * (1 + (1 << added_bits))
    return bytes_per_launch / 8 / 2 * layers


def secondary_metrics(ctx, sfntt, torch) -> dict:
    """The single-column NTT configurations: BabyBear forward + inverse for
    log n = 10..24, the M31 Circle NTT and the KoalaBear NTT likewise (n = 2^16
    is the M31 configuration), values uniform in [0, p), device-resident; 10 forward +
    inverse pairs captured in a CUDA graph, replayed 10 times after 5 warm-up
    pairs, so small sizes measure the device rather than the host's launch rate.  Columns up to 2^24 words (64 MiB) stay resident in
    the 126 MB L2 across repetitions, so the byte fraction is against HBM
    bandwidth for reference only.  Gelem/s counts n per transform."""
    res = {"note": "forward+inverse pairs on one device-resident column (L2-resident up to 2^24), "
                   "replayed from a CUDA graph"}
    stream = torch.cuda.current_stream().cuda_stream
    peak, _ = peaks()
    backends = {sfntt.FIELD_BABYBEAR: sfntt.BbCudaCtGsR4, sfntt.FIELD_M31: sfntt.CudaCtGsR4,
                sfntt.FIELD_KOALABEAR: sfntt.KbCudaCtGsR4}
    primes = {sfntt.FIELD_BABYBEAR: BB_P, sfntt.FIELD_M31: 2147483647, sfntt.FIELD_KOALABEAR: KB_P}
    fields = ((sfntt.FIELD_BABYBEAR, "bb"), (sfntt.FIELD_M31, "m31"), (sfntt.FIELD_KOALABEAR, "kb"))
    for field, name in fields:
        b = backends[field](ctx)
        rows = {}
        for log_n in range(10, 25):
            p = primes[field]
            d = torch.randint(0, p, (1 << log_n,), dtype=torch.int64, device="cuda").to(torch.int32)
            ctx.prepare(field, log_n)
            for _ in range(5):
                b.forward_dev(d.data_ptr(), log_n, 1, stream)
                b.inverse_dev(d.data_ptr(), log_n, 1, stream)
            torch.cuda.synchronize()
            # 10 pairs captured once and replayed: device time, not Python's launch rate
            graph, per_graph = torch.cuda.CUDAGraph(), 10
            with torch.cuda.graph(graph):
                cs = torch.cuda.current_stream().cuda_stream
                for _ in range(per_graph):
                    b.forward_dev(d.data_ptr(), log_n, 1, cs)
                    b.inverse_dev(d.data_ptr(), log_n, 1, cs)
            graph.replay()
            reps = 10
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                graph.replay()
            e1.record()
            torch.cuda.synchronize()
            del graph
            us = e0.elapsed_time(e1) * 1e3 / (reps * per_graph)
            n = 1 << log_n
            rows[str(log_n)] = {"fwd_inv_us": us, "gelem_s": 2 * n / (us * 1e-6) / 1e9,
                                "gbs": 16 * n / (us * 1e-6) / 1e9, "hbm_frac": 16 * n / (us * 1e-6) / 1e9 / peak}
        res[name] = rows
        best = max(rows.items(), key=lambda kv: kv[1]["gelem_s"])
        res[f"{name}_best_gelem_s"] = {"log_n": int(best[0]), "gelem_s": best[1]["gelem_s"]}
    res["m31_2^16_fwd_inv_us"] = res["m31"]["16"]["fwd_inv_us"]
    # many small columns (lattice-crypto shapes): 2^24 points per batch
    lattice = {}
    for field, name in fields:
        b = backends[field](ctx)
        for log_n in (8, 10):
            cols = 1 << (24 - log_n)
            d = torch.randint(0, BB_P, (cols << log_n,), dtype=torch.int64, device="cuda").to(torch.int32)
            ctx.prepare(field, log_n)
            for _ in range(3):
                b.forward_dev(d.data_ptr(), log_n, cols, stream)
                b.inverse_dev(d.data_ptr(), log_n, cols, stream)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(20):
                b.forward_dev(d.data_ptr(), log_n, cols, stream)
                b.inverse_dev(d.data_ptr(), log_n, cols, stream)
            e1.record()
            torch.cuda.synchronize()
            us = e0.elapsed_time(e1) * 1e3 / 20
            lattice[f"{name}_2^{log_n}x{cols}"] = {"fwd_inv_us": us, "gelem_s": 2 * (cols << log_n) / (us * 1e-6) / 1e9,
                                                   "hbm_frac": 16 * (cols << log_n) / (us * 1e-6) / 1e9 / peak}
    res["many_small_columns"] = lattice
    return res


if __name__ == "__main__":
    main()
