"""Python face of the CPU oracle (oracle/liboracle.so) — TEST INFRASTRUCTURE.

Only the test-suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline use this module; the product path never imports it. Signatures
mirror ``prism_gpu``'s so parity tests read ``oracle.f(...) == prism_gpu.f(...)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from typing import List, Optional, Sequence

import pyarrow as pa

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "prism-query_b200"))

from prism_gpu import _abi  # noqa: E402
from prism_gpu.config import (  # noqa: E402
    ARITH_F64,
    AggExpr,
    AggFunc,
    HashAggConfig,
    HashJoinConfig,
    Predicate,
    ScalarExpr,
    SortKey,
    encode_exprs,
    encode_sort_keys,
)

ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_abi.ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code
        self.kind = _abi.ERROR_NAMES.get(code, str(code))


def build_oracle() -> str:
    srcs = ["oracle.cpp", "oracle_arrow.hpp", "oracle.h"]
    newest = max(os.path.getmtime(os.path.join(ORACLE_DIR, s)) for s in srcs)
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < newest:
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return ORACLE_SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build_oracle())
        _lib.oracle_last_error.restype = C.c_char_p
        _lib.oracle_join_count_matches.restype = C.c_int64
        _lib.oracle_exact_sum_f64.restype = C.c_double
        _lib.oracle_exact_sum_f64.argtypes = [C.c_void_p, C.c_int64]
    return _lib


def _check(rc: int):
    if rc != 0:
        raise OracleError(rc, lib().oracle_last_error().decode(errors="replace"))


def _ptr_array(exported: Sequence[_abi.ExportedBatch]):
    arr = (C.POINTER(_abi.ArrowArray) * max(1, len(exported)))()
    for i, e in enumerate(exported):
        arr[i] = e.array_ptr
    return arr


def _out():
    return _abi.ArrowArray(), _abi.ArrowSchema()


def _take(a, s) -> pa.RecordBatch:
    return _abi.import_batch(a, s)


def _schema_of(batches, fallback: Optional[pa.Schema] = None):
    schema = batches[0].schema if batches else fallback
    if schema is None:
        return None, None
    es = _abi.ExportedBatch(pa.RecordBatch.from_arrays([pa.array([], type=f.type) for f in schema], schema=schema))
    return es, es.schema_ptr


DEFAULT_THREADS = 1


def hash_join(probe: pa.RecordBatch, build: pa.RecordBatch, config: HashJoinConfig, n_threads: int = DEFAULT_THREADS):
    ep, eb = _abi.ExportedBatch(probe), _abi.ExportedBatch(build)
    cfg = config.encode()
    a, s = _out()
    _check(lib().oracle_hash_join(ep.array_ptr, ep.schema_ptr, eb.array_ptr, eb.schema_ptr, C.byref(cfg), n_threads, C.byref(a), C.byref(s)))
    return _take(a, s)


def probe_matches_chunked(probes: List[pa.RecordBatch], build: pa.RecordBatch, probe_keys, build_keys, n_threads: int = DEFAULT_THREADS):
    eps = [_abi.ExportedBatch(p) for p in probes]
    eb = _abi.ExportedBatch(build)
    outs = (_abi.ArrowArray * len(probes))()
    schs = (_abi.ArrowSchema * len(probes))()
    pk, bk = _abi.int_array(probe_keys), _abi.int_array(build_keys)
    _check(lib().oracle_probe_matches_chunked(_ptr_array(eps), eps[0].schema_ptr, len(probes), eb.array_ptr, eb.schema_ptr, pk, bk, len(probe_keys), n_threads, outs, schs))
    return [_take(outs[i], schs[i]) for i in range(len(probes))]


def hash_join_probe_chunked(probes: List[pa.RecordBatch], build: pa.RecordBatch, config: HashJoinConfig, n_threads: int = DEFAULT_THREADS):
    eps = [_abi.ExportedBatch(p) for p in probes]
    eb = _abi.ExportedBatch(build)
    outs = (_abi.ArrowArray * len(probes))()
    schs = (_abi.ArrowSchema * len(probes))()
    n_out = C.c_int(0)
    cfg = config.encode()
    _check(lib().oracle_hash_join_probe_chunked(_ptr_array(eps), eps[0].schema_ptr, len(probes), eb.array_ptr, eb.schema_ptr, C.byref(cfg), n_threads, outs, schs, C.byref(n_out)))
    return [_take(outs[i], schs[i]) for i in range(n_out.value)]


def join_count_matches(probes: List[pa.RecordBatch], build: pa.RecordBatch, probe_keys, build_keys, n_threads: int, materialize: int = 1) -> int:
    eps = [_abi.ExportedBatch(p) for p in probes]
    eb = _abi.ExportedBatch(build)
    pk, bk = _abi.int_array(probe_keys), _abi.int_array(build_keys)
    r = lib().oracle_join_count_matches(_ptr_array(eps), eps[0].schema_ptr, len(probes), eb.array_ptr, eb.schema_ptr, pk, bk, len(probe_keys), n_threads, materialize)
    if r < 0:
        _check(int(-r))
    return int(r)


def hash_aggregate_batches(batches: List[pa.RecordBatch], config: HashAggConfig, n_threads: int = DEFAULT_THREADS, schema: Optional[pa.Schema] = None):
    eps = [_abi.ExportedBatch(b) for b in batches]
    es, sptr = _schema_of(batches, schema)
    cfg = config.encode()
    a, s = _out()
    _check(lib().oracle_hash_aggregate_batches(_ptr_array(eps), sptr, len(batches), C.byref(cfg), n_threads, C.byref(a), C.byref(s)))
    return _take(a, s)


def hash_aggregate(batch: pa.RecordBatch, config: HashAggConfig, n_threads: int = DEFAULT_THREADS):
    return hash_aggregate_batches([batch], config, n_threads)


def evaluate_predicate(batch: pa.RecordBatch, predicate: Predicate) -> pa.Array:
    e = _abi.ExportedBatch(batch)
    p = predicate.encode()
    a, s = _out()
    _check(lib().oracle_evaluate_predicate(e.array_ptr, e.schema_ptr, C.byref(p), C.byref(a), C.byref(s)))
    return _take(a, s).column(0)


def sort_batch(batch: pa.RecordBatch, keys: Sequence[SortKey], limit: Optional[int] = None) -> pa.RecordBatch:
    e = _abi.ExportedBatch(batch)
    k = encode_sort_keys(keys)
    a, s = _out()
    _check(lib().oracle_sort_batch(e.array_ptr, e.schema_ptr, k, len(keys), C.c_int64(-1 if limit is None else limit),
                                   C.byref(a), C.byref(s)))
    return _take(a, s)


def filter_batch(batch: pa.RecordBatch, mask: pa.Array) -> pa.RecordBatch:
    e = _abi.ExportedBatch(batch)
    m = _abi.ExportedBatch(pa.RecordBatch.from_arrays([mask], names=["mask"]))
    a, s = _out()
    _check(lib().oracle_filter_batch(e.array_ptr, e.schema_ptr, m.array_ptr, m.schema_ptr, C.byref(a), C.byref(s)))
    return _take(a, s)


def project_batch(batch: pa.RecordBatch, cols: Sequence[int]) -> pa.RecordBatch:
    e = _abi.ExportedBatch(batch)
    c = _abi.int_array(cols)
    a, s = _out()
    _check(lib().oracle_project_batch(e.array_ptr, e.schema_ptr, c, len(cols), C.byref(a), C.byref(s)))
    return _take(a, s)


def filter_and_project(batch: pa.RecordBatch, predicate: Optional[Predicate], cols: Sequence[int]) -> pa.RecordBatch:
    e = _abi.ExportedBatch(batch)
    p = predicate.encode() if predicate is not None else None
    c = _abi.int_array(cols)
    a, s = _out()
    _check(lib().oracle_filter_and_project(e.array_ptr, e.schema_ptr, C.byref(p) if p is not None else None, c, len(cols), C.byref(a), C.byref(s)))
    return _take(a, s)


def project_batch_with_exprs(batch: pa.RecordBatch, cols: Sequence[int], exprs: Sequence[ScalarExpr], arith_mode: int = ARITH_F64) -> pa.RecordBatch:
    e = _abi.ExportedBatch(batch)
    c = _abi.int_array(cols)
    ex = encode_exprs(exprs)
    a, s = _out()
    _check(lib().oracle_project_batch_with_exprs(e.array_ptr, e.schema_ptr, c, len(cols), ex, len(exprs), arith_mode, C.byref(a), C.byref(s)))
    return _take(a, s)


def evaluate_scalar_expr(batch: pa.RecordBatch, expr: ScalarExpr, arith_mode: int = ARITH_F64) -> pa.Array:
    return project_batch_with_exprs(batch, [], [expr], arith_mode).column(0)


def filter_project_aggregate(batches: List[pa.RecordBatch], predicate: Optional[Predicate], cols: Sequence[int], exprs: Sequence[ScalarExpr], agg: HashAggConfig, arith_mode: int = ARITH_F64, n_threads: int = DEFAULT_THREADS):
    eps = [_abi.ExportedBatch(b) for b in batches]
    p = predicate.encode() if predicate is not None else None
    c = _abi.int_array(cols)
    ex = encode_exprs(exprs)
    cfg = agg.encode()
    a, s = _out()
    _check(lib().oracle_filter_project_aggregate(_ptr_array(eps), eps[0].schema_ptr, len(batches), C.byref(p) if p is not None else None, c, len(cols), ex, len(exprs), arith_mode, C.byref(cfg), n_threads, C.byref(a), C.byref(s)))
    return _take(a, s)


def join_aggregate(probes: List[pa.RecordBatch], build: pa.RecordBatch, probe_keys, build_keys, cols: Sequence[int], exprs: Sequence[ScalarExpr], agg: HashAggConfig, n_threads: int = DEFAULT_THREADS):
    eps = [_abi.ExportedBatch(b) for b in probes]
    eb = _abi.ExportedBatch(build)
    pk, bk = _abi.int_array(probe_keys), _abi.int_array(build_keys)
    c = _abi.int_array(cols)
    ex = encode_exprs(exprs)
    cfg = agg.encode()
    a, s = _out()
    _check(lib().oracle_join_aggregate(_ptr_array(eps), eps[0].schema_ptr, len(probes), eb.array_ptr, eb.schema_ptr, pk, bk, len(probe_keys), c, len(cols), ex, len(exprs), C.byref(cfg), n_threads, C.byref(a), C.byref(s)))
    return _take(a, s)


# ------------------------------------------- distributed aggregation merge --
def expand_worker_aggregates(config: HashAggConfig):
    """expand_worker_aggregates (prism-bench/src/handler.rs:397-428):
    (worker config, per original aggregate the worker indices it maps to)."""
    aggs, mapping = [], []
    for a in config.aggregates:
        if a.func == AggFunc.Avg:
            i = len(aggs)
            aggs += [AggExpr(a.column, AggFunc.Sum, f"agg_{i}"), AggExpr(a.column, AggFunc.Count, f"agg_{i + 1}")]
            mapping.append([i, i + 1])
        else:
            mapping.append([len(aggs)])
            aggs.append(AggExpr(a.column, a.func, f"agg_{len(aggs)}"))
    return HashAggConfig(list(config.group_by), aggs), mapping


def _final_merge_config(nk: int, worker: HashAggConfig) -> HashAggConfig:
    """build_final_merge_config (handler.rs:430-457)."""
    def f(func):
        return func if func in (AggFunc.Min, AggFunc.Max) else AggFunc.Sum
    return HashAggConfig(list(range(nk)), [AggExpr(nk + i, f(a.func), a.output_name)
                                           for i, a in enumerate(worker.aggregates)])


def _as_f64(v) -> float:  # numeric_value_as_f64 (handler.rs:533-550): null reads 0
    return 0.0 if v is None else float(v)


def _as_i64(v) -> int:  # numeric_value_as_i64 (handler.rs:552-568): f64 `as i64` saturates, NaN -> 0
    if v is None:
        return 0
    if isinstance(v, float):
        if v != v:
            return 0
        if v >= 2.0 ** 63:
            return 2 ** 63 - 1
        if v <= -(2.0 ** 63):
            return -(2 ** 63)
        return int(v)
    return int(v)


def merge_partial_aggregates(partials: List[pa.RecordBatch], config: HashAggConfig, n_threads: int = DEFAULT_THREADS):
    """The reducer (handler.rs:327-344): hash_aggregate_batches over the
    partials with the final merge config, then
    reconstruct_original_aggregate_batch (handler.rs:459-530)."""
    nk = len(config.group_by)
    worker, mapping = expand_worker_aggregates(config)
    schema = partials[0].schema if partials else None
    merged = hash_aggregate_batches(list(partials), _final_merge_config(nk, worker), n_threads, schema=schema)
    cols = [merged.column(k) for k in range(nk)]
    fields = [merged.schema.field(k) for k in range(nk)]
    for a, m in zip(config.aggregates, mapping):
        src = merged.column(nk + m[0]).to_pylist()
        if a.func in (AggFunc.Count, AggFunc.CountDistinct):
            arr = pa.array([_as_i64(v) for v in src], type=pa.int64())
        elif a.func == AggFunc.Avg:
            cnt = merged.column(nk + m[1]).to_pylist()
            arr = pa.array([_as_f64(s) / _as_f64(c) if _as_f64(c) > 0 else 0.0 for s, c in zip(src, cnt)],
                           type=pa.float64())
        else:
            arr = pa.array([_as_f64(v) for v in src], type=pa.float64())
        cols.append(arr)
        fields.append(pa.field(a.output_name, arr.type, True))
    return pa.RecordBatch.from_arrays(cols, schema=pa.schema(fields))


# ------------------------------------------------------------- parquet ----
# The reference reads Parquet with the `parquet` crate 57.3.0 (arrow-rs),
# absent from the reference's sources; its decoding is checked here against
# pyarrow's reader (Arrow C++, an independent implementation of the same
# format), while the scan's own logic (file listing, row-group skipping,
# projection, batching, expansion) is restated from parquet_scan.rs.
def list_parquet_files(uri: str) -> List[str]:
    """list_files (object_source.rs:74-103): every *.parquet below a
    directory, or the file itself; sorted."""
    path = uri[7:] if uri.startswith("file://") else uri
    if os.path.isfile(path):
        return [path] if path.endswith(".parquet") else []
    out = []
    for root, _dirs, files in os.walk(path):
        out += [os.path.join(root, f) for f in files if f.endswith(".parquet")]
    return sorted(out)


def _check_range(v, mn, mx, op) -> bool:  # check_range / check_range_str (parquet_scan.rs:449-467)
    return {"Eq": lambda: mn <= v <= mx, "Lt": lambda: mn < v, "Le": lambda: mn <= v,
            "Gt": lambda: mx > v, "Ge": lambda: mx >= v}[op]()


# (physical type, scalar kind) -> the bounds a missing min / max defaults to
_NUMERIC_STATS = {("INT64", 1): (-2.0 ** 63, 2.0 ** 63 - 1), ("INT32", 0): (-2.0 ** 31, 2.0 ** 31 - 1),
                  ("DOUBLE", 2): (-1.7976931348623157e308, 1.7976931348623157e308)}


def _stats_might_match(pred, rg, schema_names) -> bool:
    """col_stats_might_match / stats_might_match (parquet_scan.rs:387-447)."""
    if pred.column >= len(schema_names):
        return True
    name = schema_names[pred.column]
    col = next((rg.column(i) for i in range(rg.num_columns) if rg.column(i).path_in_schema.split(".")[-1] == name), None)
    if col is None or col.statistics is None:
        return True
    st, phys, v = col.statistics, col.physical_type, pred.value
    key = (phys, v.kind)
    if key in _NUMERIC_STATS:
        lo, hi = _NUMERIC_STATS[key]
        mn = float(st.min_raw) if st.has_min_max else lo
        mx = float(st.max_raw) if st.has_min_max else hi
        return _check_range(float(v.value), mn, mx, pred.op)
    if phys == "BYTE_ARRAY" and v.kind == 3:
        if not st.has_min_max:
            return True

        def lossy(x):
            return (x if isinstance(x, bytes) else str(x).encode()).decode("utf-8", "replace").encode()
        return _check_range(v.value.encode(), lossy(st.min_raw), lossy(st.max_raw), pred.op)
    return True


def row_group_might_match(pred, rg, schema_names) -> bool:
    """row_group_might_match (parquet_scan.rs:355-377)."""
    if pred is None:
        return True
    if pred.op == "Literal":
        return bool(pred.value)
    if pred.op in ("Eq", "Lt", "Le", "Gt", "Ge"):
        return _stats_might_match(pred, rg, schema_names)
    if pred.op == "And":
        return all(row_group_might_match(c, rg, schema_names) for c in pred.children)
    if pred.op == "Or":
        return any(row_group_might_match(c, rg, schema_names) for c in pred.children)
    return True


_INT_RANGE = {pa.int8(): (-2**7, 2**7 - 1), pa.int16(): (-2**15, 2**15 - 1), pa.int32(): (-2**31, 2**31 - 1),
              pa.int64(): (-2**63, 2**63 - 1), pa.uint8(): (0, 2**8 - 1), pa.uint16(): (0, 2**16 - 1),
              pa.uint32(): (0, 2**32 - 1), pa.uint64(): (0, 2**64 - 1), pa.date32(): (-2**31, 2**31 - 1)}


def cast_safe(arr: pa.Array, typ: pa.DataType) -> pa.Array:
    """arrow_cast::cast with the default CastOptions { safe: true } (arrow-rs
    57.3.0, restated) between numeric, Boolean and Date32 types: a value the
    target cannot hold becomes null (integer range; a float truncated toward
    zero, NaN or out of range -> null), Float64 -> Float32 rounds, Boolean
    is 0 / 1, a number casts to Boolean as value != 0. Date32 casts to and
    from the integers only."""
    import numpy as np

    if arr.type == typ:
        return arr
    src = arr.type
    numeric = lambda t: pa.types.is_integer(t) or pa.types.is_floating(t) or pa.types.is_boolean(t) or t == pa.date32()  # noqa: E731
    bad_date = (src == pa.date32() or typ == pa.date32()) and (
        pa.types.is_floating(src) or pa.types.is_floating(typ) or pa.types.is_boolean(src) or pa.types.is_boolean(typ))
    if not (numeric(src) and numeric(typ)) or bad_date:
        raise OracleError(7, f"adapt_batch_to_schema: cannot cast from {src} to {typ}")
    valid = np.asarray(arr.is_valid()) if arr.null_count else np.ones(len(arr), bool)
    if pa.types.is_boolean(src):
        vals = np.asarray(arr.fill_null(False).to_numpy(zero_copy_only=False)).astype(np.int64)
        is_f = False
    elif src == pa.date32():
        vals = np.asarray(arr.cast(pa.int32()).fill_null(0).to_numpy(zero_copy_only=False)).astype(np.int64)
        is_f = False
    else:
        vals = np.asarray(arr.fill_null(0).to_numpy(zero_copy_only=False))
        is_f = pa.types.is_floating(src)
    if pa.types.is_boolean(typ):
        out = vals != 0
        return pa.array(out, type=typ, mask=~valid)
    if pa.types.is_floating(typ):
        out = vals.astype(np.float64 if typ == pa.float64() else np.float32)
        return pa.array(out, type=typ, mask=~valid)
    lo, hi = _INT_RANGE[typ]
    if is_f:
        v = vals.astype(np.float64)
        with np.errstate(invalid="ignore"):
            t = np.trunc(v)
            ok = ~np.isnan(t) & (t >= float(lo)) & (t < float(hi) + 1.0)
        iv = [int(x) if k else 0 for x, k in zip(t.tolist(), ok.tolist())]
    else:
        iv = [int(x) for x in vals.tolist()]
        ok = np.array([lo <= x <= hi for x in iv], dtype=bool) if len(iv) else np.zeros(0, bool)
        iv = [x if k else 0 for x, k in zip(iv, ok.tolist())]
    keep = valid & ok
    if typ == pa.date32():
        return pa.array(np.array(iv, dtype=np.int32), type=pa.int32(), mask=~keep).cast(pa.date32())
    return pa.array(iv, type=typ, mask=~keep)


def adapt_batch_to_schema(batch: pa.RecordBatch, target: pa.Schema) -> pa.RecordBatch:
    """adapt_batch_to_schema (parquet_scan.rs:306-339): the target's fields in
    its order, by name; another type cast (cast_safe), a missing column all
    null; RecordBatch::try_new rejects nulls in a non-nullable field."""
    cols = []
    for f in target:
        if f.name in batch.schema.names:
            c = batch.column(batch.schema.get_field_index(f.name))
            c = cast_safe(c, f.type)
        else:
            c = pa.nulls(batch.num_rows, f.type)
        if not f.nullable and c.null_count:
            raise OracleError(7, f"adapt_batch_to_schema: Column '{f.name}' is declared as non-nullable but contains null values")
        cols.append(c)
    return pa.RecordBatch.from_arrays(cols, schema=target)


def parquet_scan(uris, predicate=None, projection=None, batch_size: int = 8192, skip_expand: bool = False,
                 target_schema: pa.Schema = None):
    """parquet_scan (parquet_scan.rs:55-168) with pyarrow decoding each row group."""
    import pyarrow.parquet as pq

    files = []
    for u in uris:
        fs = list_parquet_files(u)
        if not fs:
            raise OracleError(7, f"no .parquet files found at {u}")
        files += fs
    if not files:
        return []
    full = target_schema if target_schema is not None else pq.ParquetFile(files[0]).schema_arrow
    out = []
    for f in files:
        pf = pq.ParquetFile(f)
        names = pf.schema_arrow.names
        cols = sorted({c for c in (projection or []) if 0 <= c < len(names)}) or list(range(len(names)))
        for g in range(pf.metadata.num_row_groups):
            if predicate is not None and not row_group_might_match(predicate, pf.metadata.row_group(g), names):
                continue
            t = pf.read_row_group(g, columns=[names[c] for c in cols])
            for s in range(0, t.num_rows, batch_size):
                piece = t.slice(s, batch_size).combine_chunks()
                if piece.num_rows:
                    b = piece.to_batches()[0]
                    if target_schema is not None and projection is None:  # full scans only (parquet_scan.rs:226-236)
                        b = adapt_batch_to_schema(b, target_schema)
                    out.append(b)
    if not skip_expand and projection is not None and len(projection) < len(full):
        pmap = {}
        for bi, oi in enumerate(projection):
            if 0 <= oi < len(full):
                pmap[oi] = bi
        exp = []
        for b in out:
            arrays, fields = [], []
            for i, fld in enumerate(full):
                if i in pmap:
                    c = b.column(pmap[i])
                    if c.type != fld.type:
                        raise OracleError(7, "expand batch: column types differ from the schema")
                    if not fld.nullable and c.null_count:
                        raise OracleError(7, f"expand batch: Column '{fld.name}' is declared as non-nullable but contains null values")
                    arrays.append(c)
                    fields.append(fld)
                else:
                    arrays.append(pa.nulls(b.num_rows, fld.type))
                    fields.append(pa.field(fld.name, fld.type, True))
            exp.append(pa.RecordBatch.from_arrays(arrays, schema=pa.schema(fields)))
        out = exp
    return out


def exact_sum_f64(values) -> float:
    import numpy as np

    v = np.ascontiguousarray(values, dtype=np.float64)
    return float(lib().oracle_exact_sum_f64(v.ctypes.data, len(v)))
