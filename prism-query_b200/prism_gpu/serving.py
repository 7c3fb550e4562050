"""Serving loop: operator requests of uneven sizes against resident tables.

A thin Python face of the native serving loop (prism_server_* /
prism_serve_* in include/prism_gpu.h, csrc/serve.cu): requests (a probe of a
resident hash table with device-resident int64 keys, or a GROUP BY over
device-resident columns) are submitted from any thread and answered through
futures. The native server keeps the tables resident, runs jobs on worker
threads that each own a context and CUDA stream, admits a job only while its
device footprint fits the budget, hands the smallest ready job to the next
free worker, and coalesces small requests of one shape that arrive close
together into one launch (probes of one table concatenated and cut apart by
probe row; GROUP BYs concatenated with a segment id as the first group key).
Every result equals the result of running the request alone.

This has no counterpart in the reference (its operators are called one at a
time by the Flight action handler, native/prism-flight/src/shuffle_writer.rs:294-349,
which calls QueryHandler::execute, native/prism-bench/src/handler.rs:78).
"""
from __future__ import annotations

import concurrent.futures as cf
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


class ProbeResult:
    """A probe's matches, held on the device: `matches` rows of (probe row
    of the request's keys, build payload). The tensor views are made on first
    access (making them for every result would cost each completion more
    than many small probes take on the GPU); free() releases the device
    memory now instead of when the result is garbage collected."""

    def __init__(self, matches: int, owner=None, device: int = 0, probe_rows=None, payload=None):
        self.matches = matches
        self._owner = owner   # the device batch holding the buffers
        self._device = device
        self._probe_rows = probe_rows
        self._payload = payload

    def _view(self, col: int, dtype):
        import torch

        return _device_tensor(torch, self._owner, col, dtype, self.matches, self._device)

    @property
    def probe_rows(self):
        """torch.Tensor (int32, device): the rows of the request's keys that matched."""
        if self._probe_rows is None:
            import torch

            self._probe_rows = self._view(0, torch.int32)
        return self._probe_rows

    @property
    def payload(self):
        """torch.Tensor (int64, device): the matched build rows' payload."""
        if self._payload is None:
            import torch

            self._payload = self._view(1, torch.int64)
        return self._payload

    def free(self):
        self._probe_rows = self._payload = None
        if self._owner is not None:
            self._owner.free()
            self._owner = None


@dataclass
class _Table:
    table: object        # prism_gpu.HashTable
    payload_col: int     # joined-schema column of the build payload


class Server:
    def __init__(self, device: int = 0, budget_bytes: int = 120 << 30, workers: int = 4,
                 coalesce_rows: int = 1 << 18, max_coalesce: int = 64, device_queue: bool = False,
                 queue_max_rows: int = 0, queue_ctas_per_sm: int = 0, queue_wait_limit_ms: int = 0):
        import ctypes as C

        import torch

        from . import Context, lib

        self.torch = torch
        self.device = device
        self._C = C
        self._lib = lib()
        self._ctx = Context(device)  # wraps request batches (submit side)
        self._local = threading.local()  # per completion thread: a context for exports
        self._Context = Context
        self._h = C.c_void_p()
        rc = self._lib.prism_server_create(device, budget_bytes, workers, coalesce_rows, max_coalesce, C.byref(self._h))
        if rc:
            self._raise(rc)
        if device_queue:
            # eligible probes drained by the persistent kernel (matches as a multiset)
            rc = self._lib.prism_server_set_device_queue(self._h, 1, queue_max_rows, queue_ctas_per_sm,
                                                         queue_wait_limit_ms)
            if rc:
                self._raise(rc)
        self.tables: Dict[str, int] = {}
        self._lock = threading.Lock()
        self._pending: Dict[int, tuple] = {}  # ticket -> (future, request, keepalive)
        self._submitted = 0
        self._closed = False
        # finished tickets are turned into results (export, tensor views) and
        # the futures' callbacks run on a pool as wide as the server. Every
        # thread of the pool starts now and makes its export context: a pool
        # thread started while requests run would create its context (a device
        # and a page-locked allocation, which synchronise with the device)
        # under load, stalling every worker's stream.
        self._done_pool = cf.ThreadPoolExecutor(max_workers=workers, initializer=self._init_thread)
        gate = threading.Barrier(workers)
        list(self._done_pool.map(lambda _: gate.wait(timeout=60), range(workers)))
        self._poller = threading.Thread(target=self._poll, daemon=True)
        self._poller.start()

    def _init_thread(self):
        self._local.ctx = self._Context(self.device)

    def _raise(self, rc: int):
        from . import PrismError

        msg = self._lib.prism_server_last_error(self._h) if self._h else b"server creation failed"
        raise PrismError(rc, (msg or b"").decode())

    # ------------------------------------------------------------ public --
    def register_table(self, name: str, table, payload_col: int):
        """table: a prism_gpu.HashTable (single Int64 key) the caller keeps
        alive; probes emit (probe row, build column `payload_col`)."""
        tid = self._C.c_int32(0)
        rc = self._lib.prism_server_add_table(self._h, table._h, payload_col, self._C.byref(tid))
        if rc:
            self._raise(rc)
        self.tables[name] = tid.value

    def submit(self, req) -> cf.Future:
        from . import DeviceBatch

        C = self._C
        fut: cf.Future = cf.Future()
        ticket = C.c_int64(0)
        if isinstance(req, ProbeRequest):
            keys = req.keys.contiguous()
            keep = keys
            tid = self.tables[req.table]
        else:
            n = int(req.columns[0][2].numel())
            db = DeviceBatch.from_device_buffers([(nm, f, t.data_ptr()) for nm, f, t in req.columns], n, self._ctx,
                                                 self.device)
            cfg = req.config.encode()
            keep = (db, cfg, [t for _, _, t in req.columns])
        with self._lock:  # registered before any completion can look it up
            if isinstance(req, ProbeRequest):
                rc = self._lib.prism_serve_probe(self._h, tid, keys.data_ptr(), int(keys.numel()), C.byref(ticket))
            else:
                rc = self._lib.prism_serve_aggregate(self._h, db.handle, C.byref(cfg), C.byref(ticket))
            if rc == 0:
                self._pending[ticket.value] = (fut, req, keep)
                self._submitted += 1
        if rc:
            self._raise(rc)
        return fut

    def inject_unready(self) -> cf.Future:
        """Failure injection (tests): a queued request whose descriptor never
        arrives; its future fails with Timeout once the kernel's wait runs out."""
        C = self._C
        fut: cf.Future = cf.Future()
        ticket = C.c_int64(0)
        with self._lock:
            rc = self._lib.prism_server_inject_unready(self._h, C.byref(ticket))
            if rc == 0:
                self._pending[ticket.value] = (fut, None, None)
                self._submitted += 1
        if rc:
            self._raise(rc)
        return fut

    def close(self):
        """Finishes every submitted request, then stops the native server."""
        with self._lock:
            self._closed = True
        self._poller.join()
        self._done_pool.shutdown(wait=True)
        self._lib.prism_server_destroy(self._h)
        self._h = None

    # ------------------------------------------------------------ results --
    def _poll(self):
        PRISM_ERR_TIMEOUT = 10  # include/prism_gpu.h

        C = self._C
        t = C.c_int64(0)
        taken = 0
        while True:
            rc = self._lib.prism_serve_wait_any(self._h, 20, C.byref(t))
            if rc == PRISM_ERR_TIMEOUT:
                with self._lock:
                    if self._closed and len(self._pending) == 0 and taken == self._submitted:
                        return
                continue
            taken += 1
            self._done_pool.submit(self._complete, t.value)

    def _complete(self, ticket: int):
        from . import DeviceBatch, PrismError

        C = self._C
        out = C.c_void_p()
        rc = self._lib.prism_serve_poll(self._h, ticket, 0, C.byref(out))
        with self._lock:
            fut, req, keep = self._pending.pop(ticket)
        if rc:
            msg = self._lib.prism_server_last_error(self._h)
            fut.set_exception(PrismError(rc, (msg or b"").decode()))
            return
        ctx = getattr(self._local, "ctx", None)
        if ctx is None:  # exports of different threads do not queue on one context
            ctx = self._local.ctx = self._Context(self.device)
        db = DeviceBatch(ctx, out)
        try:
            if isinstance(req, ProbeRequest):
                m = db.num_rows
                fut.set_result(ProbeResult(m, db, self.device))
            else:
                fut.set_result(db.to_arrow())
                db.free()
        except BaseException as e:  # reported on the request's future
            fut.set_exception(e)


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
                m = res.num_rows
                pr = ProbeResult(m, res, device)
                out.append(digest(len(out), pr))
                del pr
            res.free()
        else:
            n = int(r.columns[0][2].numel())
            db = DeviceBatch.from_device_buffers([(nm, f, t.data_ptr()) for nm, f, t in r.columns], n, ctx, device)
            out.append(hash_aggregate(db, r.config, ctx=ctx))
        done.append(time.perf_counter() - t0)
    return out, done
