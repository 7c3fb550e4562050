#!/usr/bin/env python
"""Benchmark: inner hash join, int64 keys (the join workload of the path).

Workload (one "step"): build a hash table over 10,000,000 build rows (unique
int64 keys = a random permutation of 0..10M, int64 payload) and probe it with
100,000,000 probe rows whose keys are Zipf(s=1.1) ranks over 1..12.5M mapped
through a seeded permutation (about 20% miss), emitting (probe_row_idx,
build_payload) for every match in the reference's order. Input rows/s =
(10M + 100M) / step time. Synthetic, seeded data of the stated shapes.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl prism|reference]
                  [--workload c2|c1|c3|c4]

--workload picks the other shapes of the path (default c2, the join above):
  c1  GROUP BY over one 1M-row batch: int64 key over 1,024 values; COUNT,
      SUM/MIN/MAX(v_i int64), SUM/AVG(v_f float64)
  c3  fused filter -> project -> aggregate over 100M fact rows (exact int128
      expressions, GROUP BY two dictionary columns)
  c4  join (15M unique utf8 build keys) -> GROUP BY over 150M probe rows

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
SCALE = 1.0
PROBE_DIST = "zipf"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--workload", choices=["c2", "c1", "c3", "c4", "c5", "sort", "topn", "parquet"], default="c2")
    ap.add_argument("--requests", type=int, default=10_000, help="c5: number of requests")
    ap.add_argument("--rate", type=float, default=2000.0, help="c5: Poisson arrival rate (requests/s)")
    ap.add_argument("--mix", choices=["both", "probe", "agg"], default="both",
                    help="c5: the request kinds (default: half GROUP BYs, half probes)")
    ap.add_argument("--max-rows", type=int, default=16_777_216, help="c5: the largest request (rows, log-uniform from 8K)")
    ap.add_argument("--queue-ctas", type=int, default=0, help="c5: persistent kernel CTAs per SM (0: the library's default)")
    ap.add_argument("--device-queue", action="store_true",
                    help="c5: probes drained by the persistent kernel's device work queue instead of the workers")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["prism", "reference"], default="prism")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--join-table", choices=["auto", "hash"], default="auto",
                    help="c2: 'auto' lets the library pick (a dense row table for the permutation keys), 'hash' "
                         "forces the open-addressing hash table")
    ap.add_argument("--partition", choices=["auto", "on", "off"], default="auto",
                    help="c2 with --join-table hash: the radix-partitioned build and probe (auto: once the hash slots "
                         "outgrow L2)")
    ap.add_argument("--probe-dist", choices=["zipf", "uniform"], default="zipf",
                    help="c2: probe keys Zipf(1.1) through a permutation (the workload) or uniform over the same "
                         "12.5M ranks (a side case without skew: every probe of a table larger than L2 misses it)")
    ap.add_argument("--tune", action="store_true",
                    help="c2 / c4 / c1: run the autotuner on the workload's own inputs first; the timed steps use "
                         "its recorded choice (reported under config.tuning)")
    ap.add_argument("--ordered", action="store_true",
                    help="c2: emit matches in the reference's probe order (default: as a multiset, one-pass probe)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="scale all sizes (profiling captures use a smaller case; bench lines use 1.0)")
    a = ap.parse_args()
    if a.join_table == "hash":
        os.environ["PRISM_JOIN_DENSE"] = "0"  # read by the library at every table build
    if a.partition != "auto":
        os.environ["PRISM_JOIN_PARTITION"] = "1" if a.partition == "on" else "0"
    if a.steps is None:
        a.steps = {"c1": 500, "c2": 200, "c3": 60, "c4": 10, "c5": 1, "sort": 10, "topn": 10, "parquet": 10}[a.workload]
    global N_BUILD, N_PROBE, ZIPF_RANKS, CPU_SAMPLE_PROBE, SCALE, PROBE_DIST, WORKLOAD
    SCALE = a.scale
    PROBE_DIST = a.probe_dist
    if PROBE_DIST == "uniform":
        WORKLOAD = WORKLOAD.replace("Zipf(1.1) int64 probe keys", "uniform int64 probe keys (over 12.5M key values)")
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
        m = min(chunk, N_PROBE - lo)
        if PROBE_DIST == "uniform":
            pkeys[lo : lo + m] = torch.randint(0, ZIPF_RANKS, (m,), generator=g, device=device, dtype=torch.int64)
            continue
        u = torch.rand(m, generator=g, device=device, dtype=torch.float64)
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


def check_c2_sample(torch, prism_gpu, ctx, build_db, bk, bp, pk, out_cols, any_order):
    """The step's output for the first 10M probe rows against the oracle's
    probe (hash_join.rs:143-200) + payload take: the (probe_row, payload)
    pairs as ordered pairs (multiset: sorted by probe row, unique build keys
    give each probe row at most one match; probe order: as emitted)."""
    import numpy as np
    import pyarrow as pa

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as oracle

    s = min(CPU_SAMPLE_PROBE, N_PROBE)
    hb = pa.RecordBatch.from_arrays([pa.array(bk.cpu().numpy()), pa.array(bp.cpu().numpy())], names=["key", "payload"])
    hpk = pk[:s].cpu().numpy()
    probes = [pa.RecordBatch.from_arrays([pa.array(hpk[i : i + 1_000_000])], names=["key"]) for i in range(0, s, 1_000_000)]
    t0 = time.perf_counter()
    pm = oracle.probe_matches_chunked(probes, hb, [0], [0], n_threads=os.cpu_count() or 1)
    ref_rows = np.concatenate([m.column(0).to_numpy().astype(np.int64) + 1_000_000 * i for i, m in enumerate(pm)])
    ref_pay = hb.column(1).to_numpy()[np.concatenate([m.column(1).to_numpy() for m in pm]).astype(np.int64)]
    dt = time.perf_counter() - t0
    sample = prism_gpu.DeviceBatch.from_device_buffers([("key", "l", pk.data_ptr())], s, ctx, pk.device.index)
    t = prism_gpu.HashTable.build(build_db, [0], ctx)
    got = t.join_project(sample, [0], [out_cols[0], 2], any_order=any_order)
    t.free()
    rows = got.column(0).to_numpy().astype(np.int64)
    pay = got.column(1).to_numpy()
    if any_order:
        o = np.argsort(rows, kind="stable")
        rows, pay = rows[o], pay[o]
    assert np.array_equal(rows, ref_rows) and np.array_equal(pay, ref_pay), "(probe_row, payload) pairs differ from the oracle"
    return (f"the first {s:,} probe rows' {len(rows):,} (probe_row, payload) pairs equal the oracle's "
            f"({'as a multiset' if any_order else 'in order'}; oracle {dt:.1f} s)")


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
    if args.workload == "c5":
        return run_c5(args, rank, world, local, torch, dist)
    if args.workload != "c2":
        return run_workload(args, rank, world, local, torch, dist)
    if args.impl == "reference":
        return run_reference(args, rank, world, torch, dist)

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import prism_gpu

    bk, bp, pk, pp = gen_c2(torch, device, seed=1234 + rank)
    torch.cuda.synchronize()
    ctx = prism_gpu.Context(local)
    # one created stream for torch's work, the events and the library (the
    # default stream's handle 0 would give the library its own stream, which
    # events on the default stream do not bracket)
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    build_db = prism_gpu.DeviceBatch.from_device_buffers([("key", "l", bk.data_ptr()), ("payload", "l", bp.data_ptr())], N_BUILD, ctx, local)
    probe_db = prism_gpu.DeviceBatch.from_device_buffers([("key", "l", pk.data_ptr()), ("payload", "i", pp.data_ptr())], N_PROBE, ctx, local)
    OUT = [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 3]
    any_order = not args.ordered
    layout = []

    def step():
        t = prism_gpu.HashTable.build(build_db, [0], ctx)
        if not layout:
            layout.append(t.layout)
        out = t.join_project(probe_db, [0], OUT, as_device=True, any_order=any_order)
        m = out.num_rows
        out.free()
        t.free()
        return m

    tuning = None
    if args.tune:
        tuning = prism_gpu.tune_join(build_db, probe_db, [0], [0], any_order=any_order, ctx=ctx)
    for _ in range(max(3, args.warmup)):
        matches = step()
    expected = int((pk < N_BUILD).sum().item())
    assert matches == expected, f"match count {matches} != {expected}"
    check = None if args.no_check else check_c2_sample(torch, prism_gpu, ctx, build_db, bk, bp, pk, OUT, any_order)

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
    # the probe phase: the one-pass probe_emit_any_kernel (matches as a
    # multiset), probe_rows_kernel + emit_rows_kernel (probe order, unique
    # int64 keys) or the single-pass probe_kernel (duplicate / general keys)
    kstats = {k: ctx.kernel_stats(k) for k in ("probe_partition_hist_kernel", "probe_partition_scatter_kernel",
                                               "probe_emit_any_kernel", "probe_rows_kernel", "emit_rows_kernel",
                                               "probe_kernel")}
    n_probe_launch = max(kstats["probe_emit_any_kernel"][0], kstats["probe_rows_kernel"][0], kstats["probe_kernel"][0])
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
    if os.path.exists(tp) and any_order and PROBE_DIST == "zipf" and not kstats["probe_partition_scatter_kernel"][0]:
        # captured for the one-pass probe on the dense table / the streamed hash probe
        traffic = json.load(open(tp)).get("probe_phase_c2" if layout[0] == "dense" else "probe_phase_c2_hash")

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
            "data": ("synthetic (seeded: permutation build keys, Zipf(1.1) probe ranks through a seeded permutation)"
                     if PROBE_DIST == "zipf" else "synthetic (seeded: permutation build keys, uniform probe keys)"),
            "config": {
                "workload": WORKLOAD,
                "build_rows": N_BUILD,
                "probe_rows": N_PROBE,
                "table": layout[0],
                "probe_path": ("radix-partitioned (keys reordered by the top 8 bits of their slot hash, then probed)"
                               if kstats["probe_partition_scatter_kernel"][0] else "streamed (probe order)"),
                "order": "any (matches as a multiset)" if any_order else "probe order (the reference's)",
                "matches_per_step": matches,
                "check": check,
                "tuning": tuning,
                "l2": "inputs larger than L2 (1.76 GB per step), no flush",
                "parallelism": f"replicated build, probe sharded (weak) x{world}",
            },
            "roofline": {
                "bound": "hbm",
                "kernel": "probe phase (" + " + ".join(k for k, v in kstats.items() if v[0]) + ")",
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


# --------------------------------------------------------------- workloads --
def sc(n):
    return max(1, int(n * SCALE))


def utf8_strings(torch, words, device):
    """Utf8 values -> (int32 offsets, uint8 data) device tensors."""
    offs = [0]
    for w in words:
        offs.append(offs[-1] + len(w.encode()))
    data = b"".join(w.encode() for w in words) or b"\0"
    return (torch.tensor(offs, dtype=torch.int32, device=device),
            torch.tensor(list(data), dtype=torch.uint8, device=device))


def pinned(torch, t):
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t)
    return h


def host_array(torch, pa, t, typ):
    h = pinned(torch, t)
    return pa.Array.from_buffers(typ, h.numel(), [None, pa.foreign_buffer(h.data_ptr(), h.numel() * h.element_size(), base=h)])


def host_utf8(torch, pa, offs, data, n):
    ho, hd = pinned(torch, offs), pinned(torch, data)
    return pa.Array.from_buffers(pa.utf8(), n, [None, pa.foreign_buffer(ho.data_ptr(), ho.numel() * 4, base=ho),
                                                pa.foreign_buffer(hd.data_ptr(), max(1, hd.numel()), base=hd)])


def host_dict(torch, pa, idx, offs, data, n_dict):
    return pa.DictionaryArray.from_arrays(host_array(torch, pa, idx, pa.int8()), host_utf8(torch, pa, offs, data, n_dict))


def oracle_mod():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py

    return oracle_py


class C1:
    """GROUP BY over one 1M-row batch (the reference's CPU-runnable case)."""
    name = "c1"
    workload = ("GROUP BY over one 1M-row batch: int64 key uniform over 1,024 values; COUNT, SUM/MIN/MAX(v_i int64), "
                "SUM/AVG(v_f float64)")
    dtype = "int64+f64"
    flush_l2 = True

    def __init__(self, torch, device, ctx, rank):
        import prism_gpu
        from prism_gpu import AggExpr, AggFunc, HashAggConfig

        self.torch, self.ctx, self.pg = torch, ctx, prism_gpu
        n = self.rows = sc(1_000_000)
        g = torch.Generator(device=device)
        g.manual_seed(100 + rank)
        keys = torch.randint(-(2**62), 2**62, (1024,), generator=g, device=device, dtype=torch.int64)
        self.key = keys[torch.randint(0, 1024, (n,), generator=g, device=device)]
        self.vi = torch.randint(-1_000_000, 1_000_001, (n,), generator=g, device=device, dtype=torch.int64)
        self.vf = torch.rand(n, generator=g, device=device, dtype=torch.float64)
        self.batch = prism_gpu.DeviceBatch.from_device_buffers(
            [("key", "l", self.key.data_ptr()), ("v_i", "l", self.vi.data_ptr()), ("v_f", "g", self.vf.data_ptr())], n, ctx,
            device.index)
        self.cfg = HashAggConfig([0], [AggExpr(0, AggFunc.Count, "count"), AggExpr(1, AggFunc.Sum, "sum_i"),
                                       AggExpr(1, AggFunc.Min, "min_i"), AggExpr(1, AggFunc.Max, "max_i"),
                                       AggExpr(2, AggFunc.Sum, "sum_f"), AggExpr(2, AggFunc.Avg, "avg_f")])

    def step(self):
        out = self.pg.hash_aggregate(self.batch, self.cfg, ctx=self.ctx, as_device=True)
        out.free()

    def tune(self):
        return self.pg.tune_hash_aggregate([self.batch], self.cfg, ctx=self.ctx)

    def host_batch(self):
        import pyarrow as pa

        t = self.torch
        schema = pa.schema([pa.field("key", pa.int64(), nullable=False), pa.field("v_i", pa.int64(), nullable=False),
                            pa.field("v_f", pa.float64(), nullable=False)])  # as the device batch declares them
        return pa.RecordBatch.from_arrays([host_array(t, pa, self.key, pa.int64()), host_array(t, pa, self.vi, pa.int64()),
                                           host_array(t, pa, self.vf, pa.float64())], schema=schema)

    def check(self):
        from helpers import assert_batches_equal

        hb = self.host_batch()
        got = self.pg.hash_aggregate(self.batch, self.cfg, ctx=self.ctx)
        ref = oracle_mod().hash_aggregate(hb, self.cfg, n_threads=1)
        assert_batches_equal(got, ref, float_cols=(4, 5, 6))
        return {"groups": got.num_rows, "full_size_check": "bit-exact vs the oracle (Float64 sums within 1e-12)"}

    def roofline(self, kstats):
        name = "agg_hash_jit" if kstats.get("agg_hash_jit", (0, 0.0))[0] else "agg_kernel"
        n, ms = kstats.get(name, (0, 0.0))
        return {"kernel": name, "bytes": 24 * self.rows, "ms": ms / max(1, n),
                "per_unit": "24 B per row (key + v_i + v_f)", "traffic_key": "agg_c1"}

    def e2e_inputs(self):
        return [self.host_batch()]

    def e2e_step(self, hb):
        return self.pg.hash_aggregate(hb[0], self.cfg, ctx=self.ctx)

    def cpu_baseline(self, threads):
        hb = self.host_batch()
        o = oracle_mod()
        o.hash_aggregate(hb, self.cfg, n_threads=1)
        runs, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < 5.0:
            o.hash_aggregate(hb, self.cfg, n_threads=1)
            runs += 1
        dt = (time.perf_counter() - t0) / runs
        return self.rows / dt, 1, (f"the whole {self.rows:,}-row batch, {runs} runs; the reference aggregates one "
                                   "RecordBatch on one thread (hash_aggregate.rs:217)")


def c3_exprs():
    from prism_gpu import ArithmeticOp, ScalarExpr, ScalarValue

    c = ScalarExpr.ColumnRef
    L = lambda v: ScalarExpr.Literal(ScalarValue.Int64(v))  # noqa: E731
    disc = ScalarExpr.BinaryOp(ArithmeticOp.Multiply, c(1), ScalarExpr.BinaryOp(ArithmeticOp.Subtract, L(100), c(2)))
    charge = ScalarExpr.BinaryOp(ArithmeticOp.Multiply, disc, ScalarExpr.BinaryOp(ArithmeticOp.Add, L(100), c(3)))
    return [disc, charge]


def c3_agg():
    from prism_gpu import AggExpr, AggFunc, HashAggConfig

    return HashAggConfig([0, 1], [
        AggExpr(2, AggFunc.Sum, "sum_disc_price"), AggExpr(2, AggFunc.Avg, "avg_disc_price"),
        AggExpr(3, AggFunc.Sum, "sum_charge"), AggExpr(3, AggFunc.Avg, "avg_charge"), AggExpr(2, AggFunc.Count, "count_order")])


class C3:
    """Fused filter -> project -> aggregate over a 100M-row fact table."""
    name = "c3"
    workload = ("fused filter->project->aggregate, 100M rows: ship_day <= 2436; price*(100-discount) and "
                "price*(100-discount)*(100+tax) exact int128 (price in cents, discount/tax in hundredths); "
                "GROUP BY (flag, status) utf8 dictionaries: SUM, AVG, COUNT")
    dtype = "int64->int128"
    flush_l2 = False

    def __init__(self, torch, device, ctx, rank):
        import prism_gpu
        from prism_gpu import Predicate, ScalarValue

        self.torch, self.ctx, self.pg = torch, ctx, prism_gpu
        n = self.rows = sc(100_000_000)
        g = torch.Generator(device=device)
        g.manual_seed(300 + rank)
        r = lambda lo, hi, dt=torch.int64: torch.randint(lo, hi, (n,), generator=g, device=device, dtype=dt)  # noqa: E731
        self.cols = {"quantity": r(1, 51), "price": r(90_000, 10_500_001), "discount": r(0, 11), "tax": r(0, 9),
                     "ship_day": r(0, 2526, torch.int32), "flag": r(0, 3, torch.int8), "status": r(0, 2, torch.int8)}
        self.fo, self.fd = utf8_strings(torch, ["A", "N", "R"], device)
        self.so, self.sd = utf8_strings(torch, ["F", "O"], device)
        c = self.cols
        self.batch = prism_gpu.DeviceBatch.from_device_buffers([
            ("quantity", "l", c["quantity"].data_ptr()), ("price", "l", c["price"].data_ptr()),
            ("discount", "l", c["discount"].data_ptr()), ("tax", "l", c["tax"].data_ptr()),
            ("ship_day", "i", c["ship_day"].data_ptr()),
            ("flag", "c", c["flag"].data_ptr(), (self.fo.data_ptr(), self.fd.data_ptr(), 3)),
            ("status", "c", c["status"].data_ptr(), (self.so.data_ptr(), self.sd.data_ptr(), 2))], n, ctx, device.index)
        self.pred = Predicate.Le(4, ScalarValue.Int32(2436))
        self.exprs, self.agg = c3_exprs(), c3_agg()

    def run(self, batches, **kw):
        return self.pg.filter_project_aggregate(batches, self.pred, [5, 6], self.exprs, self.agg,
                                                arith_mode=self.pg.ARITH_EXACT, ctx=self.ctx, **kw)

    def step(self):
        out = self.run([self.batch], as_device=True)
        out.free()

    def check(self):
        torch = self.torch
        got = self.run([self.batch])
        c = self.cols
        keep = c["ship_day"] <= 2436
        gid = c["flag"].to(torch.int64) * 2 + c["status"].to(torch.int64)
        exp = {}
        for lo in range(0, self.rows, 1_000_000):  # exact per-group sums, chunked so int64 never overflows
            sl = slice(lo, lo + 1_000_000)
            k, gg = keep[sl], gid[sl]
            disc = c["price"][sl] * (100 - c["discount"][sl])
            charge = disc * (100 + c["tax"][sl])
            for q in range(6):
                m = k & (gg == q)
                e = exp.setdefault(q, [0, 0, 0])
                e[0] += int(disc[m].sum().item())
                e[1] += int(charge[m].sum().item())
                e[2] += int(m.sum().item())
        names = {0: ("A", "F"), 1: ("A", "O"), 2: ("N", "F"), 3: ("N", "O"), 4: ("R", "F"), 5: ("R", "O")}
        cols = [got.column(i).to_pylist() for i in range(got.num_columns)]
        for row in zip(*cols):
            q = [k for k, v in names.items() if v == (row[0], row[1])][0]
            d, ch, cnt = exp[q]
            assert int(row[2]) == d and int(row[4]) == ch and row[6] == cnt, (row, exp[q])
        return {"groups": got.num_rows,
                "full_size_check": "exact int128 SUMs and COUNT per group equal chunked torch int64 sums"}

    def roofline(self, kstats):
        name = max(("agg_tiny_jit", "agg_kernel"), key=lambda k: kstats.get(k, (0, 0.0))[0])
        n, ms = kstats.get(name, (0, 0.0))
        return {"kernel": f"{name} (fused filter + project + aggregate)", "bytes": 30 * self.rows, "ms": ms / max(1, n),
                "per_unit": "30 B per row (ship_day 4 + price 8 + discount 8 + tax 8 + flag 1 + status 1)",
                "traffic_key": "agg_c3"}

    def host_batch(self, lo=0, hi=None):
        import pyarrow as pa

        t, c = self.torch, self.cols
        hi = self.rows if hi is None else hi
        sl = slice(lo, hi)
        arrs = [host_array(t, pa, c[k][sl], pa.int64()) for k in ("quantity", "price", "discount", "tax")]
        arrs.append(host_array(t, pa, c["ship_day"][sl], pa.int32()))
        arrs.append(host_dict(t, pa, c["flag"][sl], self.fo, self.fd, 3))
        arrs.append(host_dict(t, pa, c["status"][sl], self.so, self.sd, 2))
        schema = pa.schema([pa.field(nm, a.type, nullable=False) for nm, a in
                            zip(["quantity", "price", "discount", "tax", "ship_day", "flag", "status"], arrs)])
        return pa.RecordBatch.from_arrays(arrs, schema=schema)

    def e2e_inputs(self):
        return [self.host_batch()]

    def e2e_step(self, hb):
        return self.run(hb)

    def cpu_baseline(self, threads):
        o = oracle_mod()
        s = min(self.rows, 10_000_000)
        bs = [self.host_batch(lo, min(s, lo + 1_000_000)) for lo in range(0, s, 1_000_000)]
        t0 = time.perf_counter()
        o.filter_project_aggregate(bs, self.pred, [5, 6], self.exprs, self.agg, n_threads=threads)
        dt = time.perf_counter() - t0
        return s / dt, threads, (f"first {s:,} rows in 1M-row batches, the reference's Float64 expression semantics "
                                 f"({dt:.2f} s)")


class C4:
    """Join (unique utf8 build keys) -> GROUP BY over the probe stream."""
    name = "c4"
    workload = ("join->aggregate: 15M unique utf8 build keys (8-32 bytes) + int32 group id over 25 values; 150M probe "
                "rows with keys drawn Zipf(0.8) over the build keys (5% non-matching), float64 amount lognormal(5,1), "
                "in 10M-row batches; SUM(amount), COUNT GROUP BY group_id")
    dtype = "utf8+f64"
    flush_l2 = False
    BATCH = 10_000_000

    def __init__(self, torch, device, ctx, rank):
        import prism_gpu
        from prism_gpu import AggExpr, AggFunc, HashAggConfig

        self.torch, self.ctx, self.pg = torch, ctx, prism_gpu
        nb, npr = sc(15_000_000), sc(150_000_000)
        self.nb, self.np_ = nb, npr
        self.rows = nb + npr
        g = torch.Generator(device=device)
        g.manual_seed(400 + rank)
        lens = torch.randint(8, 33, (nb,), generator=g, device=device, dtype=torch.int64)
        boffs = torch.zeros(nb + 1, device=device, dtype=torch.int64)
        torch.cumsum(lens, 0, out=boffs[1:])
        bdata = torch.randint(97, 123, (int(boffs[-1].item()),), generator=g, device=device, dtype=torch.uint8)
        idx = torch.arange(nb, device=device, dtype=torch.int64)
        for k in range(6):  # the first 6 letters spell the row index in base 26: keys are unique
            bdata[boffs[:-1] + k] = (97 + (idx // 26**k) % 26).to(torch.uint8)
        self.bo32 = boffs.to(torch.int32)
        self.bdata = bdata
        self.gid = torch.randint(0, 25, (nb,), generator=g, device=device, dtype=torch.int32)
        self.build = prism_gpu.DeviceBatch.from_device_buffers(
            [("key", "u", (self.bo32.data_ptr(), bdata.data_ptr())), ("group_id", "i", self.gid.data_ptr())], nb, ctx,
            device.index)
        # Zipf(0.8) ranks over the build rows through a seeded permutation
        w = torch.arange(1, nb + 1, device=device, dtype=torch.float64).pow_(-0.8)
        cdf = torch.cumsum(w, 0)
        cdf /= cdf[-1].clone()
        del w
        perm = torch.randperm(nb, generator=g, device=device)
        self.batches, self.keep, self.hits = [], [], 0
        for lo in range(0, npr, self.BATCH):
            n = min(self.BATCH, npr - lo)
            u = torch.rand(n, generator=g, device=device, dtype=torch.float64)
            src = perm[torch.searchsorted(cdf, u, right=True).clamp_(max=nb - 1)]
            del u
            plen = lens[src]
            poffs = torch.zeros(n + 1, device=device, dtype=torch.int64)
            torch.cumsum(plen, 0, out=poffs[1:])
            row = torch.repeat_interleave(torch.arange(n, device=device), plen)
            pos = torch.arange(row.numel(), device=device) - poffs[row]
            pdata = bdata[boffs[src][row] + pos]
            del row, pos
            miss = torch.rand(n, generator=g, device=device) < 0.05
            pdata[poffs[:-1][miss]] = ord("Z")  # upper case never occurs in build keys
            self.hits += int(n - miss.sum().item())
            amount = torch.exp(5.0 + torch.randn(n, generator=g, device=device, dtype=torch.float64))  # lognormal(5, 1)
            po32 = poffs.to(torch.int32)
            del poffs, src, plen, miss
            db = prism_gpu.DeviceBatch.from_device_buffers(
                [("key", "u", (po32.data_ptr(), pdata.data_ptr())), ("amount", "g", amount.data_ptr())], n, ctx, device.index)
            self.batches.append(db)
            self.keep.append((po32, pdata, amount))
        del cdf, perm
        self.agg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "sum_amount"), AggExpr(1, AggFunc.Count, "cnt")])
        self.cols = [3, 1]  # group_id (build side), amount (probe side)

    def run(self, probes, build, **kw):
        return self.pg.join_aggregate(probes, build, [0], [0], self.cols, [], self.agg, ctx=self.ctx, **kw)

    def tune(self):
        return self.pg.tune_join_aggregate(self.batches, self.build, [0], [0], self.cols, [], self.agg, ctx=self.ctx)

    def step(self):
        out = self.run(self.batches, self.build, as_device=True)
        out.free()

    def check(self):
        got = self.run(self.batches, self.build)
        total = sum(got.column(2).to_pylist())
        assert total == self.hits, (total, self.hits)
        return {"groups": got.num_rows, "matches": self.hits,
                "full_size_check": "COUNT total == probe rows drawn from build keys"}

    def roofline(self, kstats):
        names = ("probe_kernel", "probe_rows_kernel", "emit_rows_kernel", "insert_kernel", "pack_key_records_kernel",
                 "pack_key_entries_kernel", "match_rows_kernel", "build_partition_hist_kernel", "build_partition_scatter_kernel",
                 "match_rows_kernel", "agg_kernel", "agg_tiny_jit", "agg_hash_jit", "join_agg_jit")
        ms = sum(kstats.get(k, (0, 0.0))[1] for k in names)
        steps = max(1, kstats.get("insert_kernel", (1, 0.0))[0])
        kb = int(self.bo32[-1].item()) + sum(int(k[0][-1].item()) for k in self.keep)
        nbytes = kb + 8 * self.nb + 12 * self.np_
        return {"kernel": "insert + probe + aggregation kernels (per step)", "bytes": nbytes, "ms": ms / steps,
                "per_unit": "build: key bytes + 4 B offset + 4 B group id; probe: key bytes + 4 B offset + 8 B amount",
                "traffic_key": "join_agg_c4"}

    def host_build(self):
        import pyarrow as pa

        t = self.torch
        return pa.RecordBatch.from_arrays([host_utf8(t, pa, self.bo32, self.bdata, self.nb),
                                           host_array(t, pa, self.gid, pa.int32())], names=["key", "group_id"])

    def host_probe(self, k, rows=None):
        import pyarrow as pa

        t = self.torch
        po, pd, am = self.keep[k]
        n = po.numel() - 1 if rows is None else rows
        return pa.RecordBatch.from_arrays([host_utf8(t, pa, po[: n + 1], pd, n), host_array(t, pa, am[:n], pa.float64())],
                                          names=["key", "amount"])

    def e2e_inputs(self):
        return [self.host_build()] + [self.host_probe(k) for k in range(len(self.keep))]

    def e2e_step(self, hb):
        return self.run(hb[1:], hb[0])

    def cpu_baseline(self, threads):
        o = oracle_mod()
        build = self.host_build()
        s = min(self.np_, 10_000_000)
        probes = []
        for lo in range(0, s, 1_000_000):
            pb = self.host_probe(lo // self.BATCH)
            off = lo % self.BATCH
            probes.append(pb.slice(off, min(1_000_000, s - lo)))
        t0 = time.perf_counter()
        o.join_aggregate(probes, build, [0], [0], self.cols, [], self.agg, n_threads=threads)
        dt = time.perf_counter() - t0
        return (self.nb + s) / dt, threads, (f"oracle join->aggregate: all {self.nb:,} build rows + the first {s:,} probe "
                                             f"rows in 1M-row batches ({dt:.2f} s)")


class SortW:
    """ORDER BY a Float64 key over 100M rows (sort.rs:35-78), full or top-N."""
    name = "sort"
    metric = "sort input rows/s"
    dtype = "f64 key, int64 payload"
    flush_l2 = False

    def __init__(self, torch, device, ctx, rank, limit=None):
        import prism_gpu
        from prism_gpu import NullOrdering, SortDirection, SortKey

        self.torch, self.ctx, self.pg = torch, ctx, prism_gpu
        n = self.rows = sc(100_000_000)
        self.limit = limit
        g = torch.Generator(device=device)
        g.manual_seed(600 + rank)
        self.key = torch.randn(n, generator=g, device=device, dtype=torch.float64)
        self.row = torch.arange(n, device=device, dtype=torch.int64)
        self.batch = prism_gpu.DeviceBatch.from_device_buffers(
            [("x", "g", self.key.data_ptr()), ("row", "l", self.row.data_ptr())], n, ctx, device.index)
        self.keys = [SortKey(0, SortDirection.Desc, NullOrdering.NullsLast)]
        self.workload = (f"ORDER BY x DESC{'' if limit is None else f' LIMIT {limit}'} over {n:,} rows (x float64 "
                         "normal(0,1), row int64): stable LSD radix sort, 8 passes of 8 bits, then the gather")

    def step(self):
        self.pg.sort_batch(self.batch, self.keys, limit=self.limit, ctx=self.ctx, as_device=True).free()

    def check(self):
        t = self.torch
        got = self.pg.sort_batch(self.batch, self.keys, limit=self.limit, ctx=self.ctx, as_device=True)
        m = got.num_rows
        self.ctx.synchronize()
        ptr, _, _ = got.column_device(1)
        rows = t.as_tensor(_DevView(ptr, m), device=self.key.device).clone()
        got.free()
        exp = t.sort(self.key, descending=True, stable=True).indices[:m]
        assert t.equal(rows, exp), "row order differs from torch's stable descending sort"
        return {"full_size_check": "row order equals torch.sort(descending, stable) at full size"}

    def roofline(self, kstats):
        n, ms = kstats.get("radix_scatter_kernel", (0, 0.0))
        return {"kernel": "radix_scatter_kernel (one radix pass)", "bytes": 24 * self.rows, "ms": ms / max(1, n),
                "per_unit": "24 B per row per pass (8-byte order word + 4-byte row id, read and written)",
                "traffic_key": "sort_pass"}

    def host_batch(self):
        import pyarrow as pa

        t = self.torch
        schema = pa.schema([pa.field("x", pa.float64(), nullable=False), pa.field("row", pa.int64(), nullable=False)])
        return pa.RecordBatch.from_arrays([host_array(t, pa, self.key, pa.float64()), host_array(t, pa, self.row, pa.int64())],
                                          schema=schema)

    def e2e_inputs(self):
        return [self.host_batch()]

    def e2e_step(self, hb):
        return self.pg.sort_batch(hb[0], self.keys, limit=self.limit, ctx=self.ctx)

    def cpu_baseline(self, threads):
        o = oracle_mod()
        s = min(self.rows, 10_000_000)
        hb = self.host_batch().slice(0, s)
        t0 = time.perf_counter()
        o.sort_batch(hb, self.keys, limit=self.limit)
        dt = time.perf_counter() - t0
        return s / dt, 1, (f"oracle stable sort of the first {s:,} rows on one thread (the reference sorts one "
                           f"RecordBatch with arrow's lexsort on one thread, sort.rs:35-54) ({dt:.2f} s)")


class _DevView:
    """__cuda_array_interface__ over an int64 device column another object owns."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i8", "data": (ptr, False), "version": 3}


class TopNW(SortW):
    name = "topn"

    def __init__(self, torch, device, ctx, rank):
        super().__init__(torch, device, ctx, rank, limit=100)
        self.workload = (f"ORDER BY x DESC LIMIT 100 over {self.rows:,} rows (x float64 normal(0,1), row int64): "
                         "radix select (a digit histogram of every row, then of the narrowed rows), stable sort of "
                         "the survivors, gather")

    def roofline(self, kstats):
        n, ms = kstats.get("select_hist_kernel", (0, 0.0))
        return {"kernel": "select_hist_kernel (first level: every row's top digit)", "bytes": 8 * self.rows,
                "ms": ms / max(1, n), "per_unit": "8 B per row (the Float64 key read once)", "traffic_key": "topn_select"}


class ParquetW:
    """Parquet scan (parquet_scan.rs:55-168) of a lineitem-shaped file, decoded
    on the GPU from column chunks kept compressed in HBM."""
    name = "parquet"
    metric = "parquet scan rows/s"
    dtype = "i32/i64/f64/utf8 (decoded Arrow)"
    flush_l2 = False

    def __init__(self, torch, device, ctx, rank):
        import tempfile

        import numpy as np
        import pyarrow as pa
        import pyarrow.parquet as pq

        import prism_gpu

        self.torch, self.ctx, self.pg, self.pq = torch, ctx, prism_gpu, pq
        n = self.rows = sc(30_000_000)
        rng = np.random.default_rng(700 + rank)
        flags, status = np.array(["A", "N", "R"]), np.array(["F", "O"])
        t = pa.table({
            "l_orderkey": pa.array(np.sort(rng.integers(1, 6_000_000 * 4, n))),
            "l_quantity": pa.array(rng.integers(1, 51, n).astype(np.int64)),
            "l_extendedprice": pa.array(np.round(rng.uniform(900.0, 105_000.0, n), 2)),
            "l_discount": pa.array(rng.integers(0, 11, n) / 100.0),
            "l_tax": pa.array(rng.integers(0, 9, n) / 100.0),
            "l_returnflag": pa.array(flags[rng.integers(0, 3, n)]),
            "l_linestatus": pa.array(status[rng.integers(0, 2, n)]),
            "l_shipdate": pa.array(rng.integers(8036, 10562, n).astype(np.int32), type=pa.date32()),
        })
        self.dir = tempfile.mkdtemp(prefix=f"prism_bench_pq{rank}_")
        self.path = os.path.join(self.dir, "lineitem.parquet")
        pq.write_table(t, self.path, compression="snappy", row_group_size=1 << 20)
        self.table = t
        self.prep = prism_gpu.ParquetPrepared([self.path], ctx=ctx, batch_size=1 << 20)
        self.file_bytes = os.path.getsize(self.path)
        self.decoded = int(t.nbytes)
        self.workload = (f"Parquet scan of a lineitem-shaped file: {n:,} rows x 8 columns (orderkey, quantity, "
                         "extendedprice, discount, tax, returnflag, linestatus, shipdate), written by pyarrow with its "
                         f"defaults (SNAPPY, dictionary pages with PLAIN fallback, 1 MiB pages), 1Mi-row row groups; "
                         f"{self.file_bytes / 1e6:.0f} MB on disk, {self.decoded / 1e6:.0f} MB decoded; timed: the "
                         "GPU decode of the column chunks held compressed in HBM into device batches")

    def step(self):
        for b in self.prep.decode(as_device=True):
            b.free()

    def check(self):
        got = self.pa_table(self.prep.decode())
        assert got.equals(self.table), "decoded table differs from the written one"
        return {"full_size_check": "decoded table equals the written table (every value and null)",
                "file_bytes": self.file_bytes, "compressed_bytes_in_hbm": self.prep.compressed_bytes}

    @staticmethod
    def pa_table(batches):
        import pyarrow as pa

        return pa.Table.from_batches(batches)

    def roofline(self, kstats):
        n, ms = kstats.get("pq_page_kernel", (0, 0.0))
        st = self.prep.decode(with_stats=True)[1] if not hasattr(self, "_st") else self._st
        self._st = st
        return {"kernel": "pq_page_kernel (levels, dictionary indices and PLAIN values of every page)",
                "bytes": st["inflated_bytes"] + st["decoded_bytes"], "ms": ms / max(1, n),
                "per_unit": "the inflated page bytes read + the decoded Arrow bytes written, per scan",
                "traffic_key": "parquet_page"}

    e2e_timing = ("host wall clock around prism_parquet_scan of the file (page cache warm): footer, pread of the "
                  "column chunks into pinned staging, one H2D, GPU decode, export of the batches to host Arrow (D2H)")

    def e2e_inputs(self):
        return [self.path]

    def h2d_bytes(self, _inputs):
        return self.prep.compressed_bytes

    def e2e_step(self, inputs):
        return self.pa_table(self.pg.parquet_scan(inputs, batch_size=1 << 20, ctx=self.ctx))

    def cpu_baseline(self, threads):
        t0 = time.perf_counter()
        tb = self.pq.read_table(self.path, use_threads=True)
        dt = time.perf_counter() - t0
        return tb.num_rows / dt, threads, (f"pyarrow {__import__('pyarrow').__version__} (Arrow C++) read_table of the "
                                          f"whole file on {threads} threads, page cache warm ({dt:.2f} s); the "
                                          "reference's arrow-rs parquet reader is not buildable here")


WORKLOAD_CLASSES = {"c1": C1, "c3": C3, "c4": C4, "sort": SortW, "topn": TopNW, "parquet": ParquetW}


def gpu_index_of(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if vis and vis.split(",")[local].strip().isdigit():
        return int(vis.split(",")[local])
    return local


def run_workload(args, rank, world, local, torch, dist):
    Wc = WORKLOAD_CLASSES[args.workload]
    if args.impl == "reference":
        if rank != 0:
            if world > 1:
                dist.destroy_process_group()
            return
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(0)
        import prism_gpu

        W = Wc(torch, dev, prism_gpu.Context(0), 0)
        threads = os.cpu_count() or 1
        rates = []
        for _ in range(max(1, min(args.steps, 3))):
            r, cores, sample = W.cpu_baseline(threads)
            rates.append(r)
        value = sorted(rates)[len(rates) // 2]
        line = {"metric": getattr(W, "metric", METRIC), "value": value, "unit": "rows/s", "n_gpus": world, "steps": len(rates),
                "warmup": args.warmup, "ms_per_step": W.rows / value * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": W.dtype, "data": "synthetic (seeded)", "impl": "reference",
                "config": {"workload": W.workload, "rows_per_step": W.rows},
                "cpu_baseline": {"value": value, "unit": "rows/s", "cores": cores, "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        if world > 1:
            dist.destroy_process_group()
        return

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import prism_gpu

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    ctx = prism_gpu.Context(local)
    # one created stream for torch's work, the events and the library (the
    # default stream's handle 0 would give the library its own stream, which
    # events on the default stream do not bracket)
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    W = Wc(torch, device, ctx, rank)
    torch.cuda.synchronize()
    tuning = W.tune() if args.tune and hasattr(W, "tune") else None
    for _ in range(max(3, args.warmup)):
        W.step()
    extra = {} if args.no_check else W.check()
    if tuning is not None:
        extra["tuning"] = tuning
    flush = torch.empty(256 * 1024 * 1024 // 4, device=device, dtype=torch.float32) if W.flush_l2 else None

    ctx.set_profiling(True)
    launches0 = ctx.kernel_launches
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(gpu_index_of(local)) as clocks:
        time.sleep(0.5)  # let the sampler start before the timed region
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            if flush is not None:
                flush.fill_(float(i))  # evict the inputs from L2 between steps (outside the events)
            ev[i][0].record(stream)
            W.step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    launches = ctx.kernel_launches - launches0
    names = ("probe_rows_kernel", "emit_rows_kernel", "probe_kernel", "insert_kernel", "pack_key_records_kernel",
             "pack_key_entries_kernel", "match_rows_kernel", "build_partition_hist_kernel", "build_partition_scatter_kernel", "agg_kernel", "agg_tiny_jit", "agg_hash_jit",
             "join_agg_jit", "predicate_kernel", "expr_kernel", "radix_scatter_kernel", "select_hist_kernel",
             "pq_snappy_kernel", "pq_page_kernel", "pq_copy_kernel", "pq_dict_kernel", "pq_positions_kernel")
    kstats = {k: ctx.kernel_stats(k) for k in names}
    ctx.set_profiling(False)
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * W.rows * args.steps / (ms_max / 1e3)

    rf = W.roofline(kstats)
    peak, peak_kind = peaks()
    achieved = rf["bytes"] / (rf["ms"] / 1e3) / 1e9 if rf["ms"] else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get(rf["traffic_key"])

    e2e = None
    if args.e2e_steps > 0:
        hb = W.e2e_inputs()
        h2d = W.h2d_bytes(hb) if hasattr(W, "h2d_bytes") else sum(c.nbytes for b in hb for c in b.columns)
        out = W.e2e_step(hb)  # warm
        d2h = sum(c.nbytes for c in out.columns)
        del out
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            out = W.e2e_step(hb)
            del out
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / args.e2e_steps
        tt = torch.tensor([dt], device=device, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dt = float(tt.item())
        del hb
        e2e = {"value": world * W.rows / dt, "unit": "rows/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": dt * 1e3,
               "timing": getattr(W, "e2e_timing", "host wall clock around the synchronous C-ABI calls: import (H2D "
                                 "from pinned host Arrow buffers), operator, export (D2H)")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, sample = W.cpu_baseline(os.cpu_count() or 1)
        cpu = {"value": rate, "unit": "rows/s", "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": getattr(W, "metric", METRIC), "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": W.dtype,
            "data": "synthetic (seeded torch generators with the configs' shapes and distributions)",
            "config": dict({"workload": W.workload, "rows_per_step": W.rows,
                            "l2": "L2 flushed between steps (256 MB write)" if W.flush_l2 else
                            "inputs larger than L2, no flush",
                            "parallelism": f"independent shard per GPU (weak) x{world}"}, **extra),
            "roofline": {"bound": "hbm", "kernel": rf["kernel"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                         "fallback 6650 GB/s",
                         "traffic": traffic, "algorithmic_bytes_per_launch": rf["bytes"],
                         "algorithmic_per_unit": rf["per_unit"], "avg_launch_ms": rf["ms"],
                         "kernel_ms_per_launch": {k: v[1] / v[0] for k, v in kstats.items() if v[0]}},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()



def run_c5(args, rank, world, local, torch, dist):
    """C5: a served mixed-size request stream against resident tables.

    8 resident int64 tables (log-uniform 1M-10M unique keys, built once, not
    timed per request); 10,000 requests arriving Poisson at --rate, half
    C1-style aggregations (COUNT, SUM/MIN/MAX(v_i), SUM/AVG(v_f) over 1,024
    int64 key values), half C2-style probes of a random table (keys uniform
    over 1.25x its key range: ~20% miss; emit (probe row, payload)); rows per
    request log-uniform in [8,192, 16,777,216] as slices of device-resident
    pools. Latency = arrival -> result on the host (aggregates: the result
    batch; probes: the match count, the matches staying in HBM). Compared: one
    plain launch per request in arrival order vs the serving loop (resident
    tables, admission by device footprint under a 120 GB budget, 4 worker
    streams, coalescing of small requests).
    """
    import numpy as np

    import prism_gpu
    from prism_gpu import AggExpr, AggFunc, HashAggConfig, HashTable
    from prism_gpu import serving as S

    if args.impl == "reference":
        line = {"impl": "reference", "unavailable": "the reference has no serving loop (its operators run one call at a "
                "time inside the Flight handler), so there is no reference arm for the served stream"}
        if rank == 0:
            print(json.dumps(line))
        if world > 1:
            dist.destroy_process_group()
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = prism_gpu.Context(local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    g = torch.Generator(device=dev)
    g.manual_seed(500 + rank)
    rng = np.random.default_rng(500 + rank)
    pool = sc(16_777_216)
    tables, regs, kpools = [], {}, {}
    for t in range(8):
        n = sc(int(np.exp(rng.uniform(np.log(1e6), np.log(1e7)))))
        keys = torch.randperm(n, generator=g, device=dev)
        pay = torch.randint(-(2**62), 2**62, (n,), generator=g, device=dev)
        db = prism_gpu.DeviceBatch.from_device_buffers([("k", "l", keys.data_ptr()), ("v", "l", pay.data_ptr())], n, ctx, local)
        tab = HashTable.build(db, [0], ctx)
        tables.append((tab, keys, pay, db))
        regs[f"t{t}"] = S._Table(tab, 1)
        kpools[f"t{t}"] = torch.randint(0, int(1.25 * n), (pool,), generator=g, device=dev)
    gkeys = torch.randint(-(2**62), 2**62, (1024,), generator=g, device=dev)
    akey = gkeys[torch.randint(0, 1024, (pool,), generator=g, device=dev)]
    avi = torch.randint(-1_000_000, 1_000_001, (pool,), generator=g, device=dev)
    avf = torch.rand(pool, generator=g, device=dev, dtype=torch.float64)
    cfg = HashAggConfig([0], [AggExpr(0, AggFunc.Count, "count"), AggExpr(1, AggFunc.Sum, "sum_i"),
                              AggExpr(1, AggFunc.Min, "min_i"), AggExpr(1, AggFunc.Max, "max_i"),
                              AggExpr(2, AggFunc.Sum, "sum_f"), AggExpr(2, AggFunc.Avg, "avg_f")])
    lo, hi = min(8192, pool), max(min(8192, pool), min(pool, args.max_rows))
    reqs, t = [], 0.0
    for i in range(args.requests):
        t += rng.exponential(1.0 / args.rate)
        rows = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        off = int(rng.integers(0, pool - rows + 1))
        coin = rng.random()
        if args.mix == "agg" or (args.mix == "both" and coin < 0.5):
            r = S.AggRequest([("k", "l", akey[off:off + rows]), ("vi", "l", avi[off:off + rows]),
                              ("vf", "g", avf[off:off + rows])], cfg, arrival=t)
        else:
            tn = f"t{int(rng.integers(0, 8))}"
            r = S.ProbeRequest(tn, kpools[tn][off:off + rows], arrival=t)
        reqs.append(r)
    total_rows = sum(int(r.keys.numel()) if isinstance(r, S.ProbeRequest) else int(r.columns[0][2].numel())
                     for r in reqs)
    torch.cuda.synchronize()
    # warm-up (allocator pools, every generated kernel shape, export buffers):
    # both paths on 20 requests, then the server on a burst of 200 (small
    # requests of both kinds coalesce, so the coalesced shapes compile here),
    # twice
    warm = [S.ProbeRequest(r.table, r.keys) if isinstance(r, S.ProbeRequest) else S.AggRequest(r.columns, r.config)
            for r in reqs[:200]]
    S.run_plain(warm[:20], regs, ctx, local)
    srv = S.Server(local, budget_bytes=120 << 30, workers=4, coalesce_rows=1 << 18, max_coalesce=64,
                   device_queue=args.device_queue, queue_ctas_per_sm=args.queue_ctas)
    for name, reg in regs.items():
        srv.register_table(name, reg.table, 1)
    for _ in range(2):
        [f.result() for f in [srv.submit(w) for w in warm]]

    # results: aggregates whole; probes by match count, and every 16th probe by a
    # checksum of its rows (holding every probe's output would not fit in HBM)
    def digest(i, res):
        return S.probe_digest(torch, res) if i % 16 == 1 else res.matches

    # warm-up step: the whole stream once through each path, untimed and not
    # paced, results dropped as they come; the timed passes then see the state
    # of a server that has been running (the first pass over a fresh server
    # measured 7-14 G rows/s where later passes over the same server gave
    # 15-16 G rows/s)
    def drain(rs, chunk=512):  # in chunks, so the device queue's ring never overflows
        errs = []
        for lo in range(0, len(rs), chunk):
            part = rs[lo:lo + chunk]
            left, ev, lk = [len(part)], threading.Event(), threading.Lock()

            def one(f):
                try:
                    r = f.result()
                    if isinstance(r, S.ProbeResult):
                        r.free()
                except BaseException as e:  # reported after the pass
                    errs.append(e)
                with lk:
                    left[0] -= 1
                    if left[0] == 0:
                        ev.set()

            for r in part:
                srv.submit(r).add_done_callback(one)
            ev.wait()
        if errs:
            raise errs[0]

    unpaced = [S.ProbeRequest(r.table, r.keys) if isinstance(r, S.ProbeRequest) else S.AggRequest(r.columns, r.config)
               for r in reqs]
    S.run_plain(unpaced, regs, ctx, local, digest=lambda i, res: res.matches)
    drain(unpaced)
    torch.cuda.synchronize()

    with ClockSampler(gpu_index_of(local)) as clocks:
        time.sleep(0.5)
        # the plain path: one launch per request, in arrival order
        torch.cuda.synchronize()
        plain_out, plain_done = S.run_plain(reqs, regs, ctx, local, digest=digest)
        # the served path: requests submitted at their arrival times
        done = [0.0] * len(reqs)
        served = [None] * len(reqs)
        errors, left, all_done = [], [len(reqs)], threading.Event()
        lock = threading.Lock()

        def finish(f, i):
            try:
                r = f.result()
                served[i] = digest(i, r) if isinstance(r, S.ProbeResult) else r
                if isinstance(r, S.ProbeResult):
                    r.free()  # the matches leave the device now, not when garbage collected
            except BaseException as e:  # reported after the run
                errors.append(e)
            done[i] = time.perf_counter() - t0
            with lock:
                left[0] -= 1
                if left[0] == 0:
                    all_done.set()

        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            wait = t0 + r.arrival - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            srv.submit(r).add_done_callback(lambda f, i=i: finish(f, i))
        all_done.wait()
        torch.cuda.synchronize()
    srv.close()
    if errors:
        raise errors[0]
    # every result served in the mix equals the plain (alone) one
    mism = 0
    for r, a, b in zip(reqs, plain_out, served):
        mism += int(a != b) if isinstance(r, S.ProbeRequest) else int(not a.equals(b))
    assert mism == 0, f"{mism} served results differ from the plain ones"

    def stats(done_t):
        lat = np.array([d - r.arrival for d, r in zip(done_t, reqs)]) * 1e3
        span = max(done_t) - reqs[0].arrival
        return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "rows_per_s": total_rows / span, "makespan_s": span}

    sp, ss = stats(plain_done), stats(done)
    if rank == 0:
        line = {
            "metric": "served join/agg input rows/s (p50/p99 latency beside)", "value": ss["rows_per_s"] * world,
            "unit": "rows/s", "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": ss["makespan_s"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64+f64",
            "data": "synthetic (seeded: request sizes log-uniform, Poisson arrivals, device-resident pools)",
            "config": {"workload": f"served stream: {len(reqs)} requests, Poisson {args.rate:g}/s, "
                                   + {"both": "50/50 C1-style agg / C2-style probe", "probe": "C2-style probes",
                                      "agg": "C1-style GROUP BYs"}[args.mix]
                                   + f" of 8 resident tables (1M-10M keys), rows log-uniform 8K-{hi}",
                       "total_rows": total_rows, "budget_bytes": 120 << 30, "workers": 4,
                       "device_queue": ("probes drained by one persistent kernel from a device work queue"
                                        if args.device_queue else "off (probes on the worker threads)"),
                       "l2": "request slices of 16M-row pools; most requests exceed L2",
                       "warm_up": "one untimed, unpaced pass of the whole stream through each path"},
            "served": ss, "plain_per_call": sp,
            "throughput_ratio": ss["rows_per_s"] / sp["rows_per_s"], "p99_ratio": ss["p99_ms"] / sp["p99_ms"],
            "results_equal_alone_and_in_mix": True,
            "roofline": None, "cpu_baseline": None,
            "e2e": {"value": ss["rows_per_s"] * world, "unit": "rows/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": None,
                    "timing": "arrival -> result on the host, inputs resident in HBM (the service's data)"},
            "gpu_launches": None, "clocks": clocks.summary(),
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

    any_order = not args.ordered

    def step():
        # build side up and built; the probe batch streams through the C ABI
        # in chunks whose uploads, probes and downloads overlap
        b = prism_gpu.DeviceBatch.from_arrow(hb, ctx)
        t = prism_gpu.HashTable.build(b, [0], ctx)
        out = t.join_project_arrow(hp, [0], out_cols, any_order=any_order)
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
            "ms_per_step": dt * 1e3,
            "timing": ("host wall clock around the C-ABI calls of a step: build batch import (H2D) and table build, "
                       "then prism_join_project_arrow on the host probe batch (8M-row chunks: H2D, probe and D2H "
                       "of neighbouring chunks overlap), result in host memory")}


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
