#!/usr/bin/env python
"""Benchmark: inner hash join, int64 keys (the join workload of the path).

Workload (one "step"): build a hash table over 10,000,000 build rows (unique
int64 keys = a random permutation of 0..10M, int64 payload) and probe it with
100,000,000 probe rows whose keys are Zipf(s=1.1) ranks over 1..12.5M mapped
through a seeded permutation (about 20% miss), emitting (probe_row_idx,
build_payload) for every match in the reference's order. Input rows/s =
(10M + 100M) / step time. Synthetic, seeded data of the stated shapes.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl prism|reference]

value: device-resident inputs (HBM), CUDA-event timed, max over ranks.
e2e:   the same step through the C ABI with host (pinned) Arrow buffers: H2D of
       the key/payload columns, build, probe, D2H of the result, every step.
Inputs exceed L2 (126 MB) so no flush is needed between steps.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "prism-query_b200"))

N_BUILD = 10_000_000
N_PROBE = 100_000_000
ZIPF_S = 1.1
ZIPF_RANKS = 12_500_000
METRIC = "join/agg input rows/s"
WORKLOAD = "inner hash join: 10M unique int64 build keys (+int64 payload) x 100M Zipf(1.1) int64 probe keys (+int32 payload), emit (probe_row_idx, build_payload)"
FALLBACK_HBM_GBS = 6650.0
CPU_SAMPLE_PROBE = 10_000_000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["prism", "reference"], default="prism")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="scale all sizes (profiling captures use a smaller case; bench lines use 1.0)")
    a = ap.parse_args()
    global N_BUILD, N_PROBE, ZIPF_RANKS, CPU_SAMPLE_PROBE
    if a.scale != 1.0:
        N_BUILD = int(N_BUILD * a.scale)
        N_PROBE = int(N_PROBE * a.scale)
        ZIPF_RANKS = int(ZIPF_RANKS * a.scale)
        CPU_SAMPLE_PROBE = min(CPU_SAMPLE_PROBE, N_PROBE)
    return a


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def gen_c2(torch, device, seed):
    """Seeded C2 inputs generated on the device (torch Philox generator)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    bkeys = torch.randperm(N_BUILD, generator=g, device=device, dtype=torch.int64)
    bpay = torch.randint(-(2**63), 2**63 - 1, (N_BUILD,), generator=g, device=device, dtype=torch.int64)
    w = torch.arange(1, ZIPF_RANKS + 1, device=device, dtype=torch.float64).pow_(-ZIPF_S)
    cdf = torch.cumsum(w, 0)
    cdf /= cdf[-1].clone()
    del w
    sigma = torch.randperm(ZIPF_RANKS, generator=g, device=device, dtype=torch.int64)
    pkeys = torch.empty(N_PROBE, device=device, dtype=torch.int64)
    chunk = 20_000_000
    for lo in range(0, N_PROBE, chunk):
        u = torch.rand(min(chunk, N_PROBE - lo), generator=g, device=device, dtype=torch.float64)
        r = torch.searchsorted(cdf, u, right=True).clamp_(max=ZIPF_RANKS - 1)
        pkeys[lo : lo + len(u)] = sigma[r]
        del u, r
    ppay = torch.randint(0, 2**31 - 1, (N_PROBE,), generator=g, device=device, dtype=torch.int32)
    del cdf, sigma
    return bkeys, bpay, pkeys, ppay


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200", "-i", str(self.gpu)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL,
            )
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    self.rows.append(parts)
        finally:
            os.unlink(self.path)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit())
        mx = max((float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons, "samples": len(self.rows)}


def cpu_baseline(bk, bp, pk, threads):
    """Times the oracle (a C++ restatement of hash_join.rs's build + probe +
    payload take) on the host: full 10M-row build, first 10M probe rows in
    1M-row batches probed in parallel, as the reference's rayon path does."""
    import numpy as np
    import pyarrow as pa

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as oracle

    build = pa.RecordBatch.from_arrays([pa.array(bk), pa.array(bp)], names=["key", "payload"])
    probes = [pa.RecordBatch.from_arrays([pa.array(pk[i : i + 1_000_000])], names=["key"]) for i in range(0, len(pk), 1_000_000)]
    t0 = time.perf_counter()
    m = oracle.join_count_matches(probes, build, [0], [0], threads, materialize=2)
    dt = time.perf_counter() - t0
    return (len(bk) + len(pk)) / dt, dt, m


def main():
    args = parse()
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        dist.init_process_group("nccl" if args.impl == "prism" else "gloo", timeout=datetime.timedelta(seconds=120))
    if args.impl == "reference":
        return run_reference(args, rank, world, torch, dist)

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import prism_gpu

    bk, bp, pk, pp = gen_c2(torch, device, seed=1234 + rank)
    torch.cuda.synchronize()
    ctx = prism_gpu.Context(local)
    stream = torch.cuda.current_stream(device)
    ctx.set_stream(stream.cuda_stream)
    build_db = prism_gpu.DeviceBatch.from_device_buffers([("key", "l", bk.data_ptr()), ("payload", "l", bp.data_ptr())], N_BUILD, ctx, local)
    probe_db = prism_gpu.DeviceBatch.from_device_buffers([("key", "l", pk.data_ptr()), ("payload", "i", pp.data_ptr())], N_PROBE, ctx, local)
    OUT = [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 3]

    def step():
        t = prism_gpu.HashTable.build(build_db, [0], ctx)
        out = t.join_project(probe_db, [0], OUT, as_device=True)
        m = out.num_rows
        out.free()
        t.free()
        return m

    for _ in range(max(3, args.warmup)):
        matches = step()
    expected = int((pk < N_BUILD).sum().item())
    assert matches == expected, f"match count {matches} != {expected}"

    gpu_index = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if vis and vis.split(",")[local].strip().isdigit():
        gpu_index = int(vis.split(",")[local])
    ctx.set_profiling(True)
    launches0 = ctx.kernel_launches
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_index) as clocks:
        time.sleep(0.5)  # let the sampler start before the timed region
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            step()
        stop.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = start.elapsed_time(stop)
    launches = ctx.kernel_launches - launches0
    # the probe phase: probe_rows_kernel + emit_rows_kernel (unique int64
    # keys) or the single-pass probe_kernel (duplicate / general keys)
    kstats = {k: ctx.kernel_stats(k) for k in ("probe_rows_kernel", "emit_rows_kernel", "probe_kernel")}
    n_probe_launch = max(kstats["probe_rows_kernel"][0], kstats["probe_kernel"][0])
    probe_ms = sum(v[1] for v in kstats.values())
    n_ins, ins_ms = ctx.kernel_stats("insert_kernel")
    ctx.set_profiling(False)
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    rows_per_rank = N_BUILD + N_PROBE
    value = world * rows_per_rank * args.steps / (ms_max / 1e3)

    # roofline of the dominant kernel (the probe): algorithmic bytes per launch
    # = 8 B per probe key read + 12 B per match written (u32 row + i64 payload)
    probe_bytes = 8 * N_PROBE + 12 * matches
    probe_avg_ms = probe_ms / max(1, n_probe_launch)
    achieved = probe_bytes / (probe_avg_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get("probe_phase_c2")

    # e2e: host Arrow batches in pinned memory through the C ABI
    e2e = None
    if args.e2e_steps > 0:
        e2e = run_e2e(args, torch, prism_gpu, ctx, bk, bp, pk, world, dist, device, rows_per_rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        s = CPU_SAMPLE_PROBE
        rate, dt, m = cpu_baseline(bk.cpu().numpy(), bp.cpu().numpy(), pk[:s].cpu().numpy(), threads)
        cpu = {
            "value": rate, "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": f"oracle build of all 10M build rows + probe/take of the first {s:,} probe rows in 1M-row batches ({dt:.2f} s, {m:,} matches)",
        }

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "rows/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(3, args.warmup),
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int64",
            "data": "synthetic (seeded: permutation build keys, Zipf(1.1) probe ranks through a seeded permutation)",
            "config": {
                "workload": WORKLOAD,
                "build_rows": N_BUILD,
                "probe_rows": N_PROBE,
                "matches_per_step": matches,
                "l2": "inputs larger than L2 (1.76 GB per step), no flush",
                "parallelism": f"replicated build, probe sharded (weak) x{world}",
            },
            "roofline": {
                "bound": "hbm",
                "kernel": "probe phase (probe_rows_kernel + emit_rows_kernel)",
                "kernel_ms_per_launch": {k: (v[1] / v[0] if v[0] else None) for k, v in kstats.items()},
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6650 GB/s",
                "traffic": traffic,
                "algorithmic_bytes_per_launch": probe_bytes,
                "avg_launch_ms": probe_avg_ms,
                "build_insert_ms": ins_ms / max(1, n_ins),
            },
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_e2e(args, torch, prism_gpu, ctx, bk, bp, pk, world, dist, device, rows_per_rank):
    import ctypes as C

    import pyarrow as pa

    def pinned_batch(cols):
        arrays, names, keep = [], [], []
        for name, t in cols:
            h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            h.copy_(t)
            buf = pa.foreign_buffer(h.data_ptr(), h.numel() * h.element_size(), base=h)
            typ = {torch.int64: pa.int64(), torch.int32: pa.int32()}[t.dtype]
            arrays.append(pa.Array.from_buffers(typ, h.numel(), [None, buf]))
            names.append(name)
            keep.append(h)
        return pa.RecordBatch.from_arrays(arrays, names=names), keep

    hb, keep_b = pinned_batch([("key", bk), ("payload", bp)])
    hp, keep_p = pinned_batch([("key", pk)])
    h2d = sum(c.nbytes for c in hb.columns) + sum(c.nbytes for c in hp.columns)
    out_cols = [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 2]  # probe (key) | build (key_right, payload)

    def step():
        b = prism_gpu.DeviceBatch.from_arrow(hb, ctx)
        p = prism_gpu.DeviceBatch.from_arrow(hp, ctx)
        t = prism_gpu.HashTable.build(b, [0], ctx)
        out = t.join_project(p, [0], out_cols)
        t.free()
        return out

    out = step()  # warm
    d2h = sum(c.nbytes for c in out.columns)
    del out
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        out = step()
        del out
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / args.e2e_steps
    tt = torch.tensor([dt], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    dt = float(tt.item())
    return {"value": world * rows_per_rank / dt, "unit": "rows/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": dt * 1e3, "timing": "host wall clock around synchronous C-ABI calls (import H2D, build, probe, export D2H)"}


def run_reference(args, rank, world, torch, dist):
    """The reference arm: the oracle's C++ restatement of hash_join.rs on the
    host cores (the Rust reference cannot be built here), on a bounded sample
    of the same workload per step."""
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    import numpy as np

    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    bk, bp, pk, _ = gen_c2(torch, dev, seed=1234)
    bk, bp, pk = bk.cpu().numpy(), bp.cpu().numpy(), pk[:CPU_SAMPLE_PROBE].cpu().numpy()
    threads = os.cpu_count() or 1
    for _ in range(max(1, min(args.warmup, 2))):
        cpu_baseline(bk, bp, pk, threads)
    rates = []
    for _ in range(max(1, min(args.steps, 3))):
        r, dt, m = cpu_baseline(bk, bp, pk, threads)
        rates.append(r)
    value = float(np.median(rates))
    sample = f"oracle build of 10M rows + probe/take of {CPU_SAMPLE_PROBE:,} probe rows per step, median of {len(rates)}"
    line = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": len(rates), "warmup": args.warmup,
        "ms_per_step": (N_BUILD + CPU_SAMPLE_PROBE) / value * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": WORKLOAD, "build_rows": N_BUILD, "probe_rows": N_PROBE},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
