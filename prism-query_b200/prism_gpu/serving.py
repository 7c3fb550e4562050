"""Serving loop: operator requests of uneven sizes against resident tables.

Requests arrive one by one (a probe of a resident hash table, or a GROUP BY
over a slice of device-resident rows). The server

* keeps the build-side tables resident (built once, shared by every worker);
* admits a request only while its device-memory footprint fits the budget
  (blocking admission on a byte counter);
* runs requests concurrently: each worker thread owns a context whose CUDA
  stream is its own, and the C ABI releases the GIL while the GPU works;
* hands the smallest ready job to the next free worker (shortest job
  first), so a burst of small requests is not queued behind a large one;
* coalesces small requests that arrive close together into one launch: small
  probes of one table are concatenated and probed once (each request's
  matches are the range of the output whose probe rows fall in its span —
  the output is in probe-row order); small aggregations with one config are
  concatenated with a segment-id column added as the first group key, so one
  aggregation computes every request's groups, split afterwards. Every
  request's result equals the result of running it alone: the matches are
  identical and the aggregation is exact and order-independent, its groups
  in the same first-seen order.

This has no counterpart in the reference (its operators are called one at a
time by the Flight handler, native/prism-flight/src/handler.rs).
"""
from __future__ import annotations

import concurrent.futures as cf
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import pyarrow as pa

from .config import AggExpr, HashAggConfig


@dataclass
class ProbeRequest:
    """Probe `table` with the int64 keys of a device tensor; emit (probe row, payload)."""
    table: str
    keys: object  # torch.Tensor, int64, on the server's device
    arrival: float = 0.0


@dataclass
class AggRequest:
    """GROUP BY over device-resident columns: [(name, arrow format, torch tensor)]."""
    columns: List
    config: HashAggConfig
    arrival: float = 0.0


@dataclass
class ProbeResult:
    matches: int
    probe_rows: object = None  # torch.Tensor (int32, device), rows of the request's keys, ascending
    payload: object = None     # torch.Tensor (int64, device)
    _owner: object = None      # the device batch holding the buffers


@dataclass
class _Job:
    reqs: List
    futs: List
    kind: str
    rows: int


@dataclass
class _Table:
    table: object        # prism_gpu.HashTable
    payload_col: int     # joined-schema column of the build payload


def _footprint(job: _Job) -> int:
    """Device bytes a job may hold at once: staging copy + probe words + output
    (probe) or staging + segment ids + group tables (aggregation)."""
    if job.kind == "probe":
        return job.rows * (8 + 4 + 12) + (1 << 20)
    return job.rows * (8 * 3 + 4) + (64 << 20)


class Server:
    def __init__(self, device: int = 0, budget_bytes: int = 120 << 30, workers: int = 4,
                 coalesce_rows: int = 1 << 18, max_coalesce: int = 64):
        import torch

        from . import Context

        self.torch = torch
        self.device = device
        self.budget = budget_bytes
        self.in_use = 0
        self.coalesce_rows = coalesce_rows
        self.max_coalesce = max_coalesce
        self.tables: Dict[str, _Table] = {}
        self._cv = threading.Condition()
        self._inbox: "queue.Queue" = queue.Queue()
        self._jobs: "queue.PriorityQueue" = queue.PriorityQueue()  # (rows, seq, job); smallest first
        self._seq = 0
        self._seq_lock = threading.Lock()
        self._closed = False
        self._ctxs = []
        self._threads = []
        for w in range(workers):
            ctx = Context(device)
            stream = torch.cuda.Stream(device=device)
            ctx.set_stream(stream.cuda_stream)
            self._ctxs.append((ctx, stream))
            t = threading.Thread(target=self._worker, args=(ctx, stream), daemon=True)
            t.start()
            self._threads.append(t)
        self._disp = threading.Thread(target=self._dispatch, daemon=True)
        self._disp.start()

    # ------------------------------------------------------------ public --
    def register_table(self, name: str, table, payload_col: int):
        self.tables[name] = _Table(table, payload_col)

    def submit(self, req) -> cf.Future:
        fut: cf.Future = cf.Future()
        self._inbox.put((req, fut))
        return fut

    def close(self):
        self._closed = True
        self._inbox.put(None)
        self._disp.join()
        for _ in self._threads:
            self._put(None)
        for t in self._threads:
            t.join()

    def _put(self, job: Optional[_Job]):
        """Queues a job by its row count (a closing sentinel after every job)."""
        with self._seq_lock:
            self._seq += 1
            seq = self._seq
        self._jobs.put((float("inf") if job is None else job.rows, seq, job))

    # -------------------------------------------------------- dispatcher --
    @staticmethod
    def _rows(req) -> int:
        return int(req.keys.numel()) if isinstance(req, ProbeRequest) else int(req.columns[0][2].numel())

    def _key(self, req):
        if isinstance(req, ProbeRequest):
            return ("probe", req.table)
        return ("agg", repr(req.config), tuple((n, f) for n, f, _ in req.columns))

    def _dispatch(self):
        pending: Dict[tuple, _Job] = {}
        while True:
            try:
                item = self._inbox.get(timeout=0.0005 if pending else None)
            except queue.Empty:
                item = "flush"
            if item is None:
                for j in pending.values():
                    self._put(j)
                return
            if item != "flush":
                req, fut = item
                n = self._rows(req)
                kind = "probe" if isinstance(req, ProbeRequest) else "agg"
                if n >= self.coalesce_rows:
                    self._put(_Job([req], [fut], kind, n))
                    continue
                k = self._key(req)
                j = pending.get(k)
                if j is None:
                    pending[k] = _Job([req], [fut], kind, n)
                else:
                    j.reqs.append(req)
                    j.futs.append(fut)
                    j.rows += n
                j = pending[k]
                if j.rows >= self.coalesce_rows or len(j.reqs) >= self.max_coalesce:
                    self._put(pending.pop(k))
                if not self._inbox.empty():
                    continue
            # nothing more waiting: hand over what is pending
            for k in list(pending):
                self._put(pending.pop(k))

    # ------------------------------------------------------------ worker --
    def _admit(self, nbytes: int):
        with self._cv:
            while self.in_use > 0 and self.in_use + nbytes > self.budget:
                self._cv.wait()
            self.in_use += nbytes

    def _release(self, nbytes: int):
        with self._cv:
            self.in_use -= nbytes
            self._cv.notify_all()

    def _worker(self, ctx, stream):
        torch = self.torch
        while True:
            job = self._jobs.get()[2]
            if job is None:
                return
            nbytes = _footprint(job)
            self._admit(nbytes)
            try:
                with torch.cuda.stream(stream):
                    if job.kind == "probe":
                        results = self._run_probe(ctx, stream, job.reqs)
                    else:
                        results = self._run_agg(ctx, stream, job.reqs)
                # results are read on other streams: finish this job's work first
                stream.synchronize()
                for f, r in zip(job.futs, results):
                    f.set_result(r)
            except BaseException as e:  # every request of the job fails alike
                for f in job.futs:
                    if not f.done():
                        f.set_exception(e)
            finally:
                self._release(nbytes)

    def _run_probe(self, ctx, stream, reqs: List[ProbeRequest]) -> List[ProbeResult]:
        from . import PRISM_COL_PROBE_ROW_INDEX, DeviceBatch

        torch = self.torch
        t = self.tables[reqs[0].table]
        keys = reqs[0].keys if len(reqs) == 1 else torch.cat([r.keys for r in reqs])
        n = int(keys.numel())
        db = DeviceBatch.from_device_buffers([("key", "l", keys.data_ptr())], n, ctx, self.device)
        out = t.table.join_project(db, [0], [PRISM_COL_PROBE_ROW_INDEX, 1 + t.payload_col], as_device=True, ctx=ctx)
        m = out.num_rows
        prow = _device_tensor(torch, out, 0, torch.int32, m, self.device)
        pay = _device_tensor(torch, out, 1, torch.int64, m, self.device)
        if len(reqs) == 1:
            return [ProbeResult(m, prow, pay, (out, db, keys))]
        starts = [0]
        for r in reqs:
            starts.append(starts[-1] + int(r.keys.numel()))
        bounds = torch.tensor(starts, dtype=torch.int32, device=keys.device)
        cut = torch.searchsorted(prow, bounds).cpu().tolist()  # matches are in probe-row order
        res = []
        for i in range(len(reqs)):
            a, b = cut[i], cut[i + 1]
            res.append(ProbeResult(b - a, prow[a:b] - starts[i], pay[a:b], (out, db, keys)))
        return res

    def _run_agg(self, ctx, stream, reqs: List[AggRequest]) -> List[pa.RecordBatch]:
        from . import DeviceBatch, hash_aggregate

        torch = self.torch
        cfg = reqs[0].config
        if len(reqs) == 1:
            cols = reqs[0].columns
            n = int(cols[0][2].numel())
            db = DeviceBatch.from_device_buffers([(nm, f, t.data_ptr()) for nm, f, t in cols], n, ctx, self.device)
            return [hash_aggregate(db, cfg, ctx=ctx)]
        # one aggregation for all: a segment id as the first group key
        sizes = [int(r.columns[0][2].numel()) for r in reqs]
        seg = torch.repeat_interleave(torch.arange(len(reqs), dtype=torch.int32, device=reqs[0].columns[0][2].device),
                                      torch.tensor(sizes, device=reqs[0].columns[0][2].device))
        cols = [("__segment", "i", seg)]
        for c in range(len(reqs[0].columns)):
            nm, f, _ = reqs[0].columns[c]
            cols.append((nm, f, torch.cat([r.columns[c][2] for r in reqs])))
        n = sum(sizes)
        db = DeviceBatch.from_device_buffers([(nm, f, t.data_ptr()) for nm, f, t in cols], n, ctx, self.device)
        scfg = HashAggConfig([0] + [g + 1 for g in cfg.group_by],
                             [AggExpr(a.column + 1, a.func, a.output_name) for a in cfg.aggregates])
        out = hash_aggregate(db, scfg, ctx=ctx)
        segs = out.column(0).to_numpy()
        res = []
        import numpy as np

        for i in range(len(reqs)):
            idx = np.nonzero(segs == i)[0]
            part = out.take(pa.array(idx, type=pa.int64()))
            res.append(pa.RecordBatch.from_arrays(part.columns[1:], schema=pa.schema(list(part.schema)[1:])))
        return res


class _CudaArray:
    """__cuda_array_interface__ over a device buffer another object owns."""

    def __init__(self, ptr: int, n: int, typestr: str, owner):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}
        self._owner = owner


def _device_tensor(torch, batch, col: int, dtype, n: int, device: int):
    if n == 0:
        return torch.empty(0, dtype=dtype, device=f"cuda:{device}")
    ptr, _, _ = batch.column_device(col)
    typestr = {torch.int32: "<i4", torch.int64: "<i8"}[dtype]
    return torch.as_tensor(_CudaArray(ptr, n, typestr, batch), device=f"cuda:{device}")


def probe_digest(torch, res: ProbeResult):
    """(matches, sum of probe rows, wrapping sum of payloads): a checksum of a
    probe result that equals another's when the two hold the same rows."""
    if res.matches == 0:
        return (0, 0, 0)
    return (res.matches, int(res.probe_rows.to(torch.int64).sum().item()), int(res.payload.sum().item()))


def run_plain(requests, tables: Dict[str, _Table], ctx, device: int = 0, t0: Optional[float] = None,
              digest=None):
    """The comparison path: one request at a time, in arrival order, each its
    own launch on one context; returns (results, completion times). A probe's
    result is its match count, or digest(index, ProbeResult) when given."""
    from . import PRISM_COL_PROBE_ROW_INDEX, DeviceBatch, hash_aggregate

    t0 = time.perf_counter() if t0 is None else t0
    out, done = [], []
    for r in requests:
        wait = t0 + r.arrival - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        if isinstance(r, ProbeRequest):
            t = tables[r.table]
            n = int(r.keys.numel())
            db = DeviceBatch.from_device_buffers([("key", "l", r.keys.data_ptr())], n, ctx, device)
            res = t.table.join_project(db, [0], [PRISM_COL_PROBE_ROW_INDEX, 1 + t.payload_col], as_device=True, ctx=ctx)
            if digest is None:
                out.append(res.num_rows)
            else:
                import torch

                m = res.num_rows
                pr = ProbeResult(m, _device_tensor(torch, res, 0, torch.int32, m, device),
                                 _device_tensor(torch, res, 1, torch.int64, m, device))
                out.append(digest(len(out), pr))
                del pr
            res.free()
        else:
            n = int(r.columns[0][2].numel())
            db = DeviceBatch.from_device_buffers([(nm, f, t.data_ptr()) for nm, f, t in r.columns], n, ctx, device)
            out.append(hash_aggregate(db, r.config, ctx=ctx))
        done.append(time.perf_counter() - t0)
    return out, done
