"""prism_gpu — host mirror of prism-executor's operator API over the B200 engine.

Every function here has the name, argument meaning and error behaviour of the
reference Rust function it replaces (native/prism-executor/src/lib.rs:5-15)
and runs on the GPU through the C ABI of libprism_gpu.so (include/prism_gpu.h).
There is no CPU fallback: if the CUDA library is missing or cannot reach a
device, calls raise ``PrismError``.

Batches are pyarrow ``RecordBatch``es (arrow-rs ``RecordBatch`` on the
reference side); device-resident batches are ``DeviceBatch`` handles.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass
from typing import List, Optional, Sequence

import pyarrow as pa

from . import _abi
from .config import (  # noqa: F401  (re-exported API)
    ARITH_EXACT,
    ARITH_F64,
    AggExpr,
    AggFunc,
    ArithmeticOp,
    HashAggConfig,
    HashJoinConfig,
    JoinType,
    Predicate,
    NullOrdering,
    ScalarExpr,
    ScalarValue,
    SortDirection,
    SortKey,
    encode_exprs,
    encode_sort_keys,
)

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PRISM_GPU_LIB", os.path.join(PKG_DIR, "libprism_gpu.so"))

PRISM_COL_PROBE_ROW_INDEX = -1
PRISM_JOIN_ANY_ORDER = 1  # prism_join_project_ex flag: matches as a multiset
PRISM_COL_BUILD_ROW_INDEX = -2


class PrismError(RuntimeError):
    """Mirrors PrismError (native/prism-executor/src/error.rs:6-27)."""

    def __init__(self, code: int, msg: str):
        self.code = code
        self.kind = _abi.ERROR_NAMES.get(code, str(code))
        super().__init__(f"{self.kind}: {msg}")


_lib = None
_lib_lock = threading.Lock()


def _declare(lib):
    P = C.c_void_p
    I = C.c_int
    i32 = C.c_int32
    lib.prism_ctx_create.argtypes = [I, C.c_uint64, C.POINTER(P)]
    lib.prism_ctx_destroy.argtypes = [P]
    lib.prism_ctx_destroy.restype = None
    lib.prism_last_error.argtypes = [P]
    lib.prism_last_error.restype = C.c_char_p
    lib.prism_ctx_set_stream.argtypes = [P, P]
    lib.prism_ctx_synchronize.argtypes = [P]
    lib.prism_ctx_bytes_in_use.argtypes = [P]
    lib.prism_ctx_bytes_in_use.restype = C.c_uint64
    lib.prism_ctx_kernel_launches.argtypes = [P]
    lib.prism_ctx_kernel_launches.restype = C.c_uint64
    lib.prism_version.restype = C.c_char_p
    lib.prism_ctx_set_profiling.argtypes = [P, I]
    lib.prism_ctx_kernel_stats.argtypes = [P, C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    lib.prism_jit_stats.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    lib.prism_batch_column_device.argtypes = [P, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                              C.POINTER(C.c_int32)]
    lib.prism_batch_import.argtypes = [P, P, P, C.POINTER(P)]
    lib.prism_batch_import_device.argtypes = [P, P, P, C.POINTER(P)]
    lib.prism_batch_export.argtypes = [P, P, P, P]
    lib.prism_batch_num_rows.argtypes = [P]
    lib.prism_batch_num_rows.restype = C.c_int64
    lib.prism_batch_num_columns.argtypes = [P]
    lib.prism_batch_num_columns.restype = i32
    lib.prism_batch_free.argtypes = [P]
    lib.prism_batch_free.restype = None
    lib.prism_hash_table_build.argtypes = [P, P, P, i32, C.POINTER(P)]
    lib.prism_hash_table_probe.argtypes = [P, P, P, P, i32, C.POINTER(P)]
    lib.prism_hash_table_num_rows.argtypes = [P]
    lib.prism_hash_table_num_rows.restype = C.c_int64
    lib.prism_hash_table_has_duplicates.argtypes = [P]
    lib.prism_hash_table_layout.argtypes = [P]
    lib.prism_hash_table_free.argtypes = [P]
    lib.prism_hash_table_free.restype = None
    lib.prism_join_project.argtypes = [P, P, P, P, i32, P, i32, C.POINTER(P)]
    lib.prism_join_project_ex.argtypes = [P, P, P, P, i32, P, i32, C.c_uint32, C.POINTER(P)]
    lib.prism_join_project_arrow.argtypes = [P, P, P, P, P, i32, P, i32, C.c_uint32, P, P]
    lib.prism_hash_join.argtypes = [P, P, P, P, C.POINTER(P)]
    lib.prism_probe_matches_chunked.argtypes = [P, P, i32, P, P, P, i32, P]
    lib.prism_hash_join_probe_chunked.argtypes = [P, P, i32, P, P, P, C.POINTER(i32)]
    lib.prism_hash_aggregate.argtypes = [P, P, P, C.POINTER(P)]
    lib.prism_hash_aggregate_batches.argtypes = [P, P, i32, P, C.POINTER(P)]
    lib.prism_evaluate_predicate.argtypes = [P, P, P, C.POINTER(P)]
    lib.prism_filter_batch.argtypes = [P, P, P, C.POINTER(P)]
    lib.prism_project_batch.argtypes = [P, P, P, i32, C.POINTER(P)]
    lib.prism_filter_and_project.argtypes = [P, P, P, P, i32, C.POINTER(P)]
    lib.prism_evaluate_scalar_expr.argtypes = [P, P, P, i32, C.POINTER(P)]
    lib.prism_project_batch_with_exprs.argtypes = [P, P, P, i32, P, i32, i32, C.POINTER(P)]
    lib.prism_filter_project_aggregate.argtypes = [P, P, i32, P, P, i32, P, i32, i32, P, C.POINTER(P)]
    lib.prism_join_aggregate.argtypes = [P, P, i32, P, P, P, i32, P, i32, P, i32, P, C.POINTER(P)]
    lib.prism_sort_batch.argtypes = [P, P, P, i32, C.c_int64, C.POINTER(P)]
    lib.prism_sort_batch_arrow.argtypes = [P, P, P, P, i32, C.c_int64, P, P]
    lib.prism_server_create.argtypes = [i32, C.c_uint64, i32, C.c_int64, i32, C.POINTER(P)]
    lib.prism_server_add_table.argtypes = [P, P, i32, C.POINTER(i32)]
    lib.prism_serve_probe.argtypes = [P, i32, P, C.c_int64, C.POINTER(C.c_int64)]
    lib.prism_serve_aggregate.argtypes = [P, P, P, C.POINTER(C.c_int64)]
    lib.prism_serve_poll.argtypes = [P, C.c_int64, i32, C.POINTER(P)]
    lib.prism_serve_wait_any.argtypes = [P, i32, C.POINTER(C.c_int64)]
    lib.prism_server_last_error.argtypes = [P]
    lib.prism_server_last_error.restype = C.c_char_p
    lib.prism_server_destroy.argtypes = [P]
    lib.prism_server_destroy.restype = None
    lib.prism_parquet_scan.argtypes = [P, P, C.POINTER(C.POINTER(P)), C.POINTER(i32), P]
    lib.prism_parquet_row_count.argtypes = [P, i32, P, C.POINTER(C.c_int64)]
    lib.prism_parquet_prepare.argtypes = [P, P, C.POINTER(P), P]
    lib.prism_parquet_decode.argtypes = [P, P, C.POINTER(C.POINTER(P)), C.POINTER(i32), P]
    lib.prism_parquet_prepared_rows.argtypes = [P]
    lib.prism_parquet_prepared_rows.restype = C.c_int64
    lib.prism_parquet_prepared_bytes.argtypes = [P]
    lib.prism_parquet_prepared_bytes.restype = C.c_int64
    lib.prism_parquet_prepared_free.argtypes = [P]
    lib.prism_parquet_prepared_free.restype = None
    lib.prism_free_array.argtypes = [P]
    lib.prism_free_array.restype = None
    lib.prism_expand_worker_aggregates.argtypes = [P, P, i32, C.POINTER(i32)]
    lib.prism_batch_packed_size.argtypes = [P, C.POINTER(C.c_uint64)]
    lib.prism_batch_pack.argtypes = [P, P, P, C.c_uint64]
    lib.prism_batch_unpack.argtypes = [P, P, C.c_uint64, C.POINTER(P)]
    lib.prism_arrow_packed_size.argtypes = [P, P, C.POINTER(C.c_uint64)]
    lib.prism_arrow_pack.argtypes = [P, P, P, C.c_uint64]
    lib.prism_arrow_unpack.argtypes = [P, C.c_uint64, P, P]
    lib.prism_tune_join.argtypes = [P, P, P, P, P, i32, C.c_uint32, P]
    lib.prism_server_set_device_queue.argtypes = [P, i32, C.c_int64, i32, i32]
    lib.prism_server_inject_unready.argtypes = [P, C.POINTER(C.c_int64)]
    lib.prism_tune_join_aggregate.argtypes = [P, P, i32, P, P, P, i32, P, i32, P, i32, P, P]
    lib.prism_tune_hash_aggregate.argtypes = [P, P, i32, P, P]
    lib.prism_tuning_save.argtypes = [C.c_char_p]
    lib.prism_tuning_load.argtypes = [C.c_char_p]
    lib.prism_tuning_clear.argtypes = []
    lib.prism_tuning_clear.restype = None
    lib.prism_tuning_dump.argtypes = [C.c_char_p, C.c_int64]
    lib.prism_tuning_dump.restype = C.c_int64
    lib.prism_merge_partial_aggregates.argtypes = [P, P, i32, P, C.POINTER(P)]
    lib.prism_hash_join_arrow.argtypes = [P, P, P, P, P, P, P, P]
    lib.prism_hash_aggregate_arrow.argtypes = [P, P, P, P, P, P]
    lib.prism_filter_and_project_arrow.argtypes = [P, P, P, P, P, i32, P, P]


def lib():
    """Loads libprism_gpu.so (raises PrismError if it is absent)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise PrismError(11, f"CUDA library not built: {LIB_PATH} (run __graft_entry__.build())")
            lib_ = C.CDLL(LIB_PATH)
            _declare(lib_)
            _lib = lib_
    return _lib


class Context:
    """A device context (prism_ctx): stream, allocator and counters."""

    def __init__(self, device: int = 0, memory_budget: int = 0):
        self._h = C.c_void_p()
        rc = lib().prism_ctx_create(device, memory_budget, C.byref(self._h))
        if rc != 0:
            raise PrismError(rc, "prism_ctx_create failed (no usable CUDA device?)")

    @property
    def handle(self):
        return self._h

    def check(self, rc: int):
        if rc != 0:
            msg = lib().prism_last_error(self._h)
            raise PrismError(rc, msg.decode(errors="replace") if msg else "")

    def synchronize(self):
        self.check(lib().prism_ctx_synchronize(self._h))

    def set_stream(self, stream_ptr: Optional[int]):
        self.check(lib().prism_ctx_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    @property
    def bytes_in_use(self) -> int:
        return int(lib().prism_ctx_bytes_in_use(self._h))

    @property
    def kernel_launches(self) -> int:
        return int(lib().prism_ctx_kernel_launches(self._h))

    def set_profiling(self, enable: bool):
        """Brackets the hot kernels with CUDA events (see kernel_stats)."""
        self.check(lib().prism_ctx_set_profiling(self._h, 1 if enable else 0))

    def kernel_stats(self, name: str):
        """(launches, total device ms) of kernel `name` since profiling was enabled."""
        n = C.c_uint64(0)
        ms = C.c_double(0)
        self.check(lib().prism_ctx_kernel_stats(self._h, name.encode(), C.byref(n), C.byref(ms)))
        return int(n.value), float(ms.value)

    def close(self):
        if self._h:
            lib().prism_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def jit_stats():
    """(enabled, compiles, total compile ms) of the run-time kernel compiler."""
    e, n, ms = C.c_int32(0), C.c_int64(0), C.c_double(0)
    lib().prism_jit_stats(C.byref(e), C.byref(n), C.byref(ms))
    return bool(e.value), int(n.value), float(ms.value)


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(int(os.environ.get("PRISM_GPU_DEVICE", "0")))
    return _default_ctx


class DeviceBatch:
    """A device-resident RecordBatch (prism_batch)."""

    def __init__(self, ctx: Context, handle: C.c_void_p, keepalive=None):
        self.ctx = ctx
        self._h = handle
        self._keep = keepalive

    @staticmethod
    def from_arrow(batch: pa.RecordBatch, ctx: Optional[Context] = None) -> "DeviceBatch":
        ctx = ctx or default_context()
        e = _abi.ExportedBatch(batch)
        h = C.c_void_p()
        ctx.check(lib().prism_batch_import(ctx.handle, e.array_ptr, e.schema_ptr, C.byref(h)))
        e.release()
        return DeviceBatch(ctx, h)

    @staticmethod
    def from_device_buffers(columns, num_rows: int, ctx: Optional[Context] = None, device_id: int = 0) -> "DeviceBatch":
        """Wraps device-resident, null-free columns without a copy.

        columns: list of
          (name, arrow_format, values_ptr)                 fixed width
          (name, "u", (offsets_ptr, data_ptr))              Utf8 (int32 offsets)
          (name, index_format, indices_ptr, (dict_offsets_ptr, dict_data_ptr, dict_len))
                                                           Utf8 dictionary
        The memory must outlive the batch (e.g. torch tensors the caller keeps).
        """
        ctx = ctx or default_context()
        keep = []
        n = len(columns)
        child_arrays = (C.POINTER(_abi.ArrowArray) * n)()
        child_schemas = (C.POINTER(_abi.ArrowSchema) * n)()
        for i, col in enumerate(columns):
            name, fmt, ptr = col[0], col[1], col[2]
            nm, fm = name.encode(), fmt.encode()
            dict_a = dict_s = None
            if fmt == "u":
                offs, data = ptr
                bufs = (C.c_void_p * 3)(None, offs, data)
                nbuf = 3
            else:
                bufs = (C.c_void_p * 2)(None, ptr)
                nbuf = 2
                if len(col) > 3:
                    doffs, ddata, dlen = col[3]
                    dbufs = (C.c_void_p * 3)(None, doffs, ddata)
                    da = _abi.ArrowArray(dlen, 0, 0, 3, 0, dbufs, None, None)
                    ds = _abi.ArrowSchema(b"u", b"", None, 0, 0, None, None)
                    keep += [dbufs, da, ds]
                    dict_a, dict_s = C.pointer(da), C.pointer(ds)
            a = _abi.ArrowArray(num_rows, 0, 0, nbuf, 0, bufs, None, dict_a)
            s_ = _abi.ArrowSchema(fm, nm, None, 0, 0, None, dict_s)
            keep += [bufs, a, s_, nm, fm]
            child_arrays[i] = C.pointer(a)
            child_schemas[i] = C.pointer(s_)
        top_bufs = (C.c_void_p * 1)(None)
        dev = _abi.ArrowDeviceArray()
        dev.array = _abi.ArrowArray(num_rows, 0, 0, 1, n, top_bufs, child_arrays, None)
        dev.device_id = device_id
        dev.device_type = _abi.ARROW_DEVICE_CUDA
        sch = _abi.ArrowSchema(b"+s", b"", None, 0, n, child_schemas, None)
        keep += [top_bufs, child_arrays, child_schemas]
        h = C.c_void_p()
        ctx.check(lib().prism_batch_import_device(ctx.handle, C.byref(dev), C.byref(sch), C.byref(h)))
        return DeviceBatch(ctx, h, keepalive=keep)

    @property
    def handle(self):
        return self._h

    @property
    def num_rows(self) -> int:
        return int(lib().prism_batch_num_rows(self._h))

    @property
    def num_columns(self) -> int:
        return int(lib().prism_batch_num_columns(self._h))

    def column_device(self, col: int):
        """(values pointer, validity pointer or 0, element width) of column
        `col` in device memory, without a copy; valid while the batch lives."""
        v, m, w = C.c_void_p(), C.c_void_p(), C.c_int32(0)
        self.ctx.check(lib().prism_batch_column_device(self._h, col, C.byref(v), C.byref(m), C.byref(w)))
        return int(v.value or 0), int(m.value or 0), int(w.value)

    def packed_size(self) -> int:
        """Bytes of this batch in the packed form (prism_batch_pack)."""
        n = C.c_uint64(0)
        rc = lib().prism_batch_packed_size(self._h, C.byref(n))
        if rc:
            raise PrismError(rc, (lib().prism_last_error(None) or b"").decode())
        return int(n.value)

    def pack_into(self, device_ptr: int, capacity: int):
        """Writes the packed batch to device memory at `device_ptr`
        (stream-ordered on the context's stream)."""
        self.ctx.check(lib().prism_batch_pack(self.ctx.handle, self._h, C.c_void_p(device_ptr), capacity))

    @staticmethod
    def unpack(device_ptr: int, size: int, ctx: Optional[Context] = None) -> "DeviceBatch":
        """A batch read from a packed device buffer (the payload is copied)."""
        ctx = ctx or default_context()
        h = C.c_void_p()
        ctx.check(lib().prism_batch_unpack(ctx.handle, C.c_void_p(device_ptr), size, C.byref(h)))
        return DeviceBatch(ctx, h)

    def to_arrow(self) -> pa.RecordBatch:
        a, s = _abi.ArrowArray(), _abi.ArrowSchema()
        self.ctx.check(lib().prism_batch_export(self.ctx.handle, self._h, C.byref(a), C.byref(s)))
        return _abi.import_batch(a, s)

    def free(self):
        if self._h:
            lib().prism_batch_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _dev(batch, ctx) -> DeviceBatch:
    if isinstance(batch, DeviceBatch):
        return batch
    return DeviceBatch.from_arrow(batch, ctx)


def _ptrs(batches: Sequence[DeviceBatch]):
    arr = (C.c_void_p * max(1, len(batches)))()
    for i, b in enumerate(batches):
        arr[i] = b.handle
    return arr


def _result(ctx, h, as_device: bool):
    db = DeviceBatch(ctx, h)
    return db if as_device else db.to_arrow()


# ------------------------------------------------------------ hash join ----


@dataclass
class ProbeMatches:
    """hash_join.rs:67-70."""

    probe_indices: pa.Array
    build_indices: pa.Array


class HashTable:
    """Resident build-side table (HashTable, hash_join.rs:77-201)."""

    def __init__(self, ctx: Context, handle, build: DeviceBatch):
        self.ctx = ctx
        self._h = handle
        self._build = build

    @staticmethod
    def build(batch, key_cols: Sequence[int], ctx: Optional[Context] = None) -> "HashTable":
        ctx = ctx or default_context()
        db = _dev(batch, ctx)
        keys = _abi.int_array(key_cols)
        h = C.c_void_p()
        ctx.check(lib().prism_hash_table_build(ctx.handle, db.handle, keys, len(key_cols), C.byref(h)))
        return HashTable(ctx, h, db)

    def probe(self, probe_batch, probe_key_cols: Sequence[int], as_device=False):
        db = _dev(probe_batch, self.ctx)
        keys = _abi.int_array(probe_key_cols)
        h = C.c_void_p()
        self.ctx.check(lib().prism_hash_table_probe(self.ctx.handle, self._h, db.handle, keys, len(probe_key_cols), C.byref(h)))
        out = _result(self.ctx, h, as_device)
        if as_device:
            return out
        return out.column(0), out.column(1)

    def join_project(self, probe_batch, probe_key_cols: Sequence[int], out_cols: Sequence[int], as_device=False,
                     ctx: Optional[Context] = None, any_order: bool = False):
        """Probe and gather `out_cols` of the joined schema (PRISM_COL_* for
        row indices). `ctx` (default: the table's) picks the context, hence
        the stream, the probe runs on: a resident table serves any context of
        its device. `any_order`: the matches as a multiset (one-pass probe)."""
        ctx = ctx or self.ctx
        db = _dev(probe_batch, ctx)
        keys = _abi.int_array(probe_key_cols)
        oc = _abi.int_array(out_cols)
        h = C.c_void_p()
        ctx.check(lib().prism_join_project_ex(ctx.handle, self._h, db.handle, keys, len(probe_key_cols), oc,
                                              len(out_cols), PRISM_JOIN_ANY_ORDER if any_order else 0, C.byref(h)))
        return _result(ctx, h, as_device)

    def join_project_arrow(self, probe_batch: pa.RecordBatch, probe_key_cols: Sequence[int], out_cols: Sequence[int],
                           any_order: bool = False, ctx: Optional[Context] = None) -> pa.RecordBatch:
        """join_project with a host probe batch and a host result, through
        prism_join_project_arrow (streamed in chunks: uploads, probes and
        downloads overlap)."""
        ctx = ctx or self.ctx
        e = _abi.ExportedBatch(probe_batch)
        keys = _abi.int_array(probe_key_cols)
        oc = _abi.int_array(out_cols)
        a, s = _abi.ArrowArray(), _abi.ArrowSchema()
        try:
            ctx.check(lib().prism_join_project_arrow(ctx.handle, self._h, e.array_ptr, e.schema_ptr, keys,
                                                     len(probe_key_cols), oc, len(out_cols),
                                                     PRISM_JOIN_ANY_ORDER if any_order else 0, C.byref(a), C.byref(s)))
        finally:
            e.release()
        return _abi.import_batch(a, s)

    @property
    def has_duplicates(self) -> bool:
        return bool(lib().prism_hash_table_has_duplicates(self._h))

    @property
    def layout(self) -> str:
        """'hash' (open-addressing slots) or 'dense' (a row per key value)."""
        return {0: "hash", 1: "dense"}.get(lib().prism_hash_table_layout(self._h), "unknown")

    def free(self):
        if self._h:
            lib().prism_hash_table_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def hash_join(probe_batch, build_batch, config: HashJoinConfig, ctx: Optional[Context] = None, as_device=False):
    """hash_join (hash_join.rs:312-365)."""
    ctx = ctx or default_context()
    p, b = _dev(probe_batch, ctx), _dev(build_batch, ctx)
    cfg = config.encode()
    h = C.c_void_p()
    ctx.check(lib().prism_hash_join(ctx.handle, p.handle, b.handle, C.byref(cfg), C.byref(h)))
    return _result(ctx, h, as_device)


def probe_matches_chunked(probe_batches, build_batch, probe_key_cols, build_key_cols, ctx: Optional[Context] = None) -> List[ProbeMatches]:
    """probe_matches_chunked (hash_join.rs:286-309)."""
    ctx = ctx or default_context()
    ps = [_dev(p, ctx) for p in probe_batches]
    b = _dev(build_batch, ctx)
    outs = (C.c_void_p * max(1, len(ps)))()
    pk, bk = _abi.int_array(probe_key_cols), _abi.int_array(build_key_cols)
    ctx.check(lib().prism_probe_matches_chunked(ctx.handle, _ptrs(ps), len(ps), b.handle, pk, bk, len(probe_key_cols), outs))
    res = []
    for i in range(len(ps)):
        rb = DeviceBatch(ctx, C.c_void_p(outs[i])).to_arrow()
        res.append(ProbeMatches(rb.column(0), rb.column(1)))
    return res


def hash_join_probe_chunked(probe_batches, build_batch, config: HashJoinConfig, ctx: Optional[Context] = None) -> List[pa.RecordBatch]:
    """hash_join_probe_chunked (hash_join.rs:206-282)."""
    ctx = ctx or default_context()
    ps = [_dev(p, ctx) for p in probe_batches]
    b = _dev(build_batch, ctx)
    outs = (C.c_void_p * max(1, len(ps)))()
    n_out = C.c_int32(0)
    cfg = config.encode()
    ctx.check(lib().prism_hash_join_probe_chunked(ctx.handle, _ptrs(ps), len(ps), b.handle, C.byref(cfg), outs, C.byref(n_out)))
    return [DeviceBatch(ctx, C.c_void_p(outs[i])).to_arrow() for i in range(n_out.value)]


# ------------------------------------------------------------ aggregate ----


def hash_aggregate_batches(batches, config: HashAggConfig, ctx: Optional[Context] = None, as_device=False):
    """hash_aggregate_batches (hash_aggregate.rs:182-339)."""
    ctx = ctx or default_context()
    ds = [_dev(b, ctx) for b in batches]
    cfg = config.encode()
    h = C.c_void_p()
    ctx.check(lib().prism_hash_aggregate_batches(ctx.handle, _ptrs(ds), len(ds), C.byref(cfg), C.byref(h)))
    return _result(ctx, h, as_device)


def hash_aggregate(batch, config: HashAggConfig, ctx: Optional[Context] = None, as_device=False):
    """hash_aggregate (hash_aggregate.rs:174-176)."""
    ctx = ctx or default_context()
    d = _dev(batch, ctx)
    cfg = config.encode()
    h = C.c_void_p()
    ctx.check(lib().prism_hash_aggregate(ctx.handle, d.handle, C.byref(cfg), C.byref(h)))
    return _result(ctx, h, as_device)


# ------------------------------------------------------------ parquet ----


def _uri_array(uris: Sequence[str]):
    enc = [os.fspath(u).encode() for u in uris]
    arr = (C.c_char_p * max(1, len(enc)))(*enc)
    return arr, enc


def _scan_config(uris, predicate, projection, batch_size, skip_expand, target_schema=None):
    arr, keep = _uri_array(uris)
    pred = predicate.encode() if predicate is not None else None
    proj = _abi.int_array(list(projection)) if projection is not None else None
    ts = None
    if target_schema is not None:  # exported through the C Data Interface (released with the config)
        ts = _abi.ExportedSchema(target_schema)
    cfg = _abi.prism_parquet_scan_config(arr, len(keep), C.cast(C.pointer(pred), C.c_void_p) if pred is not None else None,
                                         proj, len(projection) if projection is not None else 0, batch_size,
                                         1 if skip_expand else 0, C.cast(ts.schema_ptr, C.c_void_p) if ts else None)
    cfg._keep = (arr, keep, pred, proj, ts)
    return cfg


def _batch_list(ctx, out, n, as_device):
    try:
        return [_result(ctx, C.c_void_p(out[i]), as_device) for i in range(n.value)]
    finally:
        lib().prism_free_array(C.cast(out, C.c_void_p))


def _stats_dict(st):
    return {f: getattr(st, f) for f, _ in st._fields_}


def parquet_scan(uris: Sequence[str], predicate: Optional[Predicate] = None, projection: Optional[Sequence[int]] = None,
                 batch_size: int = 8192, skip_expand: bool = False, ctx: Optional[Context] = None, as_device=False,
                 with_stats=False, target_schema: Optional[pa.Schema] = None):
    """parquet_scan (parquet_scan.rs:55-168), decoded on the GPU: a list of
    batches (Arrow, or DeviceBatch with as_device); with_stats also returns
    the scan's counters (files, row groups read / skipped, pages, bytes).
    target_schema: ParquetScanConfig.target_schema (schema evolution)."""
    ctx = ctx or default_context()
    cfg = _scan_config(uris, predicate, projection, batch_size, skip_expand, target_schema)
    out = C.POINTER(C.c_void_p)()
    n = C.c_int32(0)
    st = _abi.prism_parquet_scan_stats()
    ctx.check(lib().prism_parquet_scan(ctx.handle, C.byref(cfg), C.byref(out), C.byref(n), C.byref(st)))
    res = _batch_list(ctx, out, n, as_device)
    return (res, _stats_dict(st)) if with_stats else res


class ParquetPrepared:
    """A Parquet scan's column chunks kept in HBM still compressed
    (prism_parquet_prepare); decode() runs the GPU decoder over them."""

    def __init__(self, uris: Sequence[str], predicate: Optional[Predicate] = None,
                 projection: Optional[Sequence[int]] = None, batch_size: int = 8192, skip_expand: bool = False,
                 ctx: Optional[Context] = None, target_schema: Optional[pa.Schema] = None):
        self.ctx = ctx or default_context()
        cfg = _scan_config(uris, predicate, projection, batch_size, skip_expand, target_schema)
        h = C.c_void_p()
        st = _abi.prism_parquet_scan_stats()
        self.ctx.check(lib().prism_parquet_prepare(self.ctx.handle, C.byref(cfg), C.byref(h), C.byref(st)))
        self._h = h
        self.stats = _stats_dict(st)

    @property
    def num_rows(self) -> int:
        return int(lib().prism_parquet_prepared_rows(self._h))

    @property
    def compressed_bytes(self) -> int:
        return int(lib().prism_parquet_prepared_bytes(self._h))

    def decode(self, as_device=False, with_stats=False):
        out = C.POINTER(C.c_void_p)()
        n = C.c_int32(0)
        st = _abi.prism_parquet_scan_stats()
        self.ctx.check(lib().prism_parquet_decode(self.ctx.handle, self._h, C.byref(out), C.byref(n), C.byref(st)))
        res = _batch_list(self.ctx, out, n, as_device)
        return (res, _stats_dict(st)) if with_stats else res

    def free(self):
        if self._h:
            lib().prism_parquet_prepared_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def parquet_row_count(uris: Sequence[str], predicate: Optional[Predicate] = None) -> int:
    """parquet_row_count (parquet_scan.rs:240-266), from the footers alone."""
    arr, keep = _uri_array(uris)
    pred = predicate.encode() if predicate is not None else None
    n = C.c_int64(0)
    rc = lib().prism_parquet_row_count(arr, len(keep), C.byref(pred) if pred is not None else None, C.byref(n))
    if rc:
        raise PrismError(rc, (lib().prism_last_error(None) or b"").decode())
    return int(n.value)


def expand_worker_aggregates(config: HashAggConfig) -> HashAggConfig:
    """The worker-side config of a distributed aggregation
    (expand_worker_aggregates, prism-bench/src/handler.rs:397-428): AVG
    becomes SUM then COUNT of its column, every other aggregate stays; the
    outputs are named agg_<i>."""
    cfg = config.encode()
    out = (_abi.prism_agg_expr * max(1, 2 * len(config.aggregates)))()
    n = C.c_int32(0)
    rc = lib().prism_expand_worker_aggregates(C.byref(cfg), out, 2 * len(config.aggregates), C.byref(n))
    if rc:
        raise PrismError(rc, (lib().prism_last_error(None) or b"").decode())
    aggs = [AggExpr(out[i].column, AggFunc(out[i].func), out[i].output_name.decode()) for i in range(n.value)]
    return HashAggConfig(list(config.group_by), aggs)


def pack_arrow(batch: pa.RecordBatch) -> bytearray:
    """A host batch in the packed exchange format (prism_arrow_pack): the
    same bytes prism_batch_pack writes for the batch on a device."""
    e = _abi.ExportedBatch(batch)
    try:
        n = C.c_uint64(0)
        rc = lib().prism_arrow_packed_size(e.array_ptr, e.schema_ptr, C.byref(n))
        if rc:
            raise PrismError(rc, (lib().prism_last_error(None) or b"").decode())
        buf = bytearray(int(n.value))
        cbuf = (C.c_char * len(buf)).from_buffer(buf)
        rc = lib().prism_arrow_pack(e.array_ptr, e.schema_ptr, C.addressof(cbuf), len(buf))
        if rc:
            raise PrismError(rc, (lib().prism_last_error(None) or b"").decode())
        del cbuf
        return buf
    finally:
        e.release()


def unpack_arrow(data) -> pa.RecordBatch:
    """A packed batch (host bytes, from either pack) as a host batch
    (prism_arrow_unpack; the result owns a copy)."""
    mv = memoryview(data).cast("B")
    if mv.readonly:
        mv = memoryview(bytearray(mv))
    cbuf = (C.c_char * len(mv)).from_buffer(mv)
    a, s = _abi.ArrowArray(), _abi.ArrowSchema()
    rc = lib().prism_arrow_unpack(C.addressof(cbuf), len(mv), C.byref(a), C.byref(s))
    del cbuf
    if rc:
        raise PrismError(rc, (lib().prism_last_error(None) or b"").decode())
    return _abi.import_batch(a, s)


def merge_partial_aggregates(partials, config: HashAggConfig, ctx: Optional[Context] = None, as_device=False):
    """The reducer merge of per-worker partial aggregates
    (prism-bench/src/handler.rs:327-344) on the GPU: `partials` (Arrow or
    device batches, reducer's own first) are outputs of
    expand_worker_aggregates(config); the result has config's columns."""
    ctx = ctx or default_context()
    ds = [_dev(b, ctx) for b in partials]
    cfg = config.encode()
    h = C.c_void_p()
    ctx.check(lib().prism_merge_partial_aggregates(ctx.handle, _ptrs(ds), len(ds), C.byref(cfg), C.byref(h)))
    return _result(ctx, h, as_device)


# ------------------------------------------------------- filter / project --


def evaluate_predicate(batch, predicate: Predicate, ctx: Optional[Context] = None) -> pa.Array:
    """evaluate_predicate (filter_project.rs:65-123)."""
    ctx = ctx or default_context()
    d = _dev(batch, ctx)
    p = predicate.encode()
    h = C.c_void_p()
    ctx.check(lib().prism_evaluate_predicate(ctx.handle, d.handle, C.byref(p), C.byref(h)))
    return DeviceBatch(ctx, h).to_arrow().column(0)


def sort_batch(batch, keys: Sequence[SortKey], limit: Optional[int] = None, ctx: Optional[Context] = None,
               as_device=False):
    """sort_batch / sort_batch_limit (sort.rs:35-78): the rows ordered by
    `keys` (most significant first), the first `limit` of them when given.
    topn_single_col (sort.rs:97-146) is a Float64 Desc key with a limit."""
    ctx = ctx or default_context()
    d = _dev(batch, ctx)
    k = encode_sort_keys(keys)
    h = C.c_void_p()
    ctx.check(lib().prism_sort_batch(ctx.handle, d.handle, k, len(keys), -1 if limit is None else int(limit),
                                     C.byref(h)))
    return _result(ctx, h, as_device)


def filter_batch(batch, mask, ctx: Optional[Context] = None, as_device=False):
    """filter_batch (filter_project.rs:126-135)."""
    ctx = ctx or default_context()
    d = _dev(batch, ctx)
    if isinstance(mask, DeviceBatch):
        m = mask
    else:
        m = DeviceBatch.from_arrow(pa.RecordBatch.from_arrays([mask], names=["mask"]), ctx)
    h = C.c_void_p()
    ctx.check(lib().prism_filter_batch(ctx.handle, d.handle, m.handle, C.byref(h)))
    return _result(ctx, h, as_device)


def project_batch(batch, column_indices: Sequence[int], ctx: Optional[Context] = None, as_device=False):
    """project_batch (filter_project.rs:138-160)."""
    ctx = ctx or default_context()
    d = _dev(batch, ctx)
    c = _abi.int_array(column_indices)
    h = C.c_void_p()
    ctx.check(lib().prism_project_batch(ctx.handle, d.handle, c, len(column_indices), C.byref(h)))
    return _result(ctx, h, as_device)


def filter_and_project(batch, predicate: Optional[Predicate], column_indices: Sequence[int], ctx: Optional[Context] = None, as_device=False):
    """filter_and_project (filter_project.rs:163-180)."""
    ctx = ctx or default_context()
    d = _dev(batch, ctx)
    p = predicate.encode() if predicate is not None else None
    c = _abi.int_array(column_indices)
    h = C.c_void_p()
    ctx.check(lib().prism_filter_and_project(ctx.handle, d.handle, C.byref(p) if p is not None else None, c, len(column_indices), C.byref(h)))
    return _result(ctx, h, as_device)


def evaluate_scalar_expr(batch, expr: ScalarExpr, arith_mode: int = ARITH_F64, ctx: Optional[Context] = None) -> pa.Array:
    """evaluate_scalar_expr (filter_project.rs:216-294)."""
    ctx = ctx or default_context()
    d = _dev(batch, ctx)
    e = expr.encode()
    h = C.c_void_p()
    ctx.check(lib().prism_evaluate_scalar_expr(ctx.handle, d.handle, C.byref(e), arith_mode, C.byref(h)))
    return DeviceBatch(ctx, h).to_arrow().column(0)


def project_batch_with_exprs(batch, column_indices: Sequence[int], expressions: Sequence[ScalarExpr], arith_mode: int = ARITH_F64, ctx: Optional[Context] = None, as_device=False):
    """project_batch_with_exprs (filter_project.rs:305-333)."""
    ctx = ctx or default_context()
    d = _dev(batch, ctx)
    c = _abi.int_array(column_indices)
    ex = encode_exprs(expressions)
    h = C.c_void_p()
    ctx.check(lib().prism_project_batch_with_exprs(ctx.handle, d.handle, c, len(column_indices), ex, len(expressions), arith_mode, C.byref(h)))
    return _result(ctx, h, as_device)


# ------------------------------------------------------------------ fused --


def filter_project_aggregate(batches, predicate: Optional[Predicate], column_indices: Sequence[int], expressions: Sequence[ScalarExpr], agg: HashAggConfig, arith_mode: int = ARITH_F64, ctx: Optional[Context] = None, as_device=False):
    """Filter -> project -> aggregate in one pass (executor.rs:91-186 node chain)."""
    ctx = ctx or default_context()
    ds = [_dev(b, ctx) for b in batches]
    p = predicate.encode() if predicate is not None else None
    c = _abi.int_array(column_indices)
    ex = encode_exprs(expressions)
    cfg = agg.encode()
    h = C.c_void_p()
    ctx.check(
        lib().prism_filter_project_aggregate(
            ctx.handle, _ptrs(ds), len(ds), C.byref(p) if p is not None else None, c, len(column_indices), ex, len(expressions), arith_mode, C.byref(cfg), C.byref(h)
        )
    )
    return _result(ctx, h, as_device)


def join_aggregate(probe_batches, build_batch, probe_keys, build_keys, column_indices: Sequence[int], expressions: Sequence[ScalarExpr], agg: HashAggConfig, ctx: Optional[Context] = None, as_device=False):
    """Fused inner join -> project -> aggregate (executor.rs:333-458)."""
    ctx = ctx or default_context()
    ps = [_dev(b, ctx) for b in probe_batches]
    b = _dev(build_batch, ctx)
    pk, bk = _abi.int_array(probe_keys), _abi.int_array(build_keys)
    c = _abi.int_array(column_indices)
    ex = encode_exprs(expressions)
    cfg = agg.encode()
    h = C.c_void_p()
    ctx.check(
        lib().prism_join_aggregate(
            ctx.handle, _ptrs(ps), len(ps), b.handle, pk, bk, len(probe_keys), c, len(column_indices), ex, len(expressions), C.byref(cfg), C.byref(h)
        )
    )
    return _result(ctx, h, as_device)


# ------------------------------------------------------------- autotuner ----
def tune_join(build_batch, probe_batch, build_keys: Sequence[int], probe_keys: Sequence[int], any_order: bool = False,
              ctx: Optional[Context] = None) -> dict:
    """Times the join table settings on this build / probe pair and records
    the fastest for the build side's shape class (prism_tune_join)."""
    ctx = ctx or default_context()
    b, p = _dev(build_batch, ctx), _dev(probe_batch, ctx)
    r = _abi.TuneResult()
    ctx.check(lib().prism_tune_join(ctx.handle, b.handle, p.handle, _abi.int_array(build_keys), _abi.int_array(probe_keys),
                                    len(build_keys), PRISM_JOIN_ANY_ORDER if any_order else 0, C.byref(r)))
    return r.as_dict()


def tune_join_aggregate(probe_batches, build_batch, probe_keys, build_keys, column_indices: Sequence[int],
                        expressions: Sequence[ScalarExpr], agg: HashAggConfig, ctx: Optional[Context] = None) -> dict:
    """Times the fused join -> aggregate kernel shapes on these inputs and
    records the fastest for the build side's shape class."""
    ctx = ctx or default_context()
    ps = [_dev(b, ctx) for b in probe_batches]
    b = _dev(build_batch, ctx)
    cfg = agg.encode()
    r = _abi.TuneResult()
    ctx.check(lib().prism_tune_join_aggregate(
        ctx.handle, _ptrs(ps), len(ps), b.handle, _abi.int_array(probe_keys), _abi.int_array(build_keys), len(probe_keys),
        _abi.int_array(column_indices), len(column_indices), encode_exprs(expressions), len(expressions), C.byref(cfg),
        C.byref(r)))
    return r.as_dict()


def tune_hash_aggregate(batches, config: HashAggConfig, ctx: Optional[Context] = None) -> dict:
    """Times the hashed-groups kernel's block sizes on these batches and
    records the fastest for their row-count class."""
    ctx = ctx or default_context()
    ds = [_dev(b, ctx) for b in batches]
    cfg = config.encode()
    r = _abi.TuneResult()
    ctx.check(lib().prism_tune_hash_aggregate(ctx.handle, _ptrs(ds), len(ds), C.byref(cfg), C.byref(r)))
    return r.as_dict()


def tuning_save(path: str):
    rc = lib().prism_tuning_save(path.encode())
    if rc:
        raise PrismError(rc, (lib().prism_last_error(None) or b"").decode())


def tuning_load(path: str):
    rc = lib().prism_tuning_load(path.encode())
    if rc:
        raise PrismError(rc, (lib().prism_last_error(None) or b"").decode())


def tuning_clear():
    lib().prism_tuning_clear()


def tuning_dump() -> str:
    n = lib().prism_tuning_dump(None, 0)
    buf = C.create_string_buffer(n + 1)
    lib().prism_tuning_dump(buf, n + 1)
    return buf.value.decode()
