"""Comparison helpers shared by the parity tests."""
from __future__ import annotations

import math

import numpy as np
import pyarrow as pa

# Float64 SUM/AVG tolerance against the reference's sequential f64 sums
FLOAT_RTOL = 1e-12


def _is_float(t: pa.DataType) -> bool:
    return pa.types.is_floating(t)


def assert_batches_equal(got: pa.RecordBatch, ref: pa.RecordBatch, float_cols=(), rtol: float = FLOAT_RTOL):
    """Schemas identical; integer/byte/key columns bit-exact; columns listed in
    float_cols (by index) within rtol (NaN matches NaN, +-inf exact)."""
    assert got.schema.names == ref.schema.names, (got.schema.names, ref.schema.names)
    for i, (fg, fr) in enumerate(zip(got.schema, ref.schema)):
        assert fg.type == fr.type, (i, fg, fr)
        assert fg.nullable == fr.nullable, (i, fg, fr)
    assert got.num_rows == ref.num_rows, (got.num_rows, ref.num_rows)
    for i in range(got.num_columns):
        a, b = got.column(i), ref.column(i)
        if i in float_cols and _is_float(a.type):
            assert a.null_count == b.null_count
            x = a.to_numpy(zero_copy_only=False)
            y = b.to_numpy(zero_copy_only=False)
            close(x, y, rtol)
        else:
            if pa.types.is_dictionary(a.type):
                assert a.to_pylist() == b.to_pylist(), f"column {i}"
            elif _is_float(a.type):
                # bit-exact, with NaN equal to NaN (pyarrow's equals is not)
                assert a.null_count == b.null_count, f"column {i} null count"
                va = np.asarray(a.is_valid()) if a.null_count else np.ones(len(a), bool)
                vb = np.asarray(b.is_valid()) if b.null_count else np.ones(len(b), bool)
                assert np.array_equal(va, vb), f"column {i} validity"
                x = a.to_numpy(zero_copy_only=False)[va]
                y = b.to_numpy(zero_copy_only=False)[vb]
                same = (x == y) | (np.isnan(x) & np.isnan(y))
                assert same.all(), f"column {i} ({got.schema.names[i]}) differs at {np.flatnonzero(~same)[:5]}"
                sx = np.signbit(x[~np.isnan(x)])
                sy = np.signbit(y[~np.isnan(y)])
                assert np.array_equal(sx, sy), f"column {i} signed-zero mismatch"
            else:
                assert a.equals(b), f"column {i} ({got.schema.names[i]}) differs:\n{a}\n{b}"


def close(x, y, rtol=FLOAT_RTOL):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    assert x.shape == y.shape
    both_nan = np.isnan(x) & np.isnan(y)
    fin = np.isfinite(x) & np.isfinite(y)
    assert np.all(both_nan | fin | (x == y)), "non-finite mismatch"
    d = np.abs(x[fin] - y[fin])
    tol = rtol * np.maximum(np.abs(y[fin]), np.finfo(np.float64).tiny)
    bad = d > tol
    assert not bad.any(), f"{bad.sum()} values beyond rtol {rtol}: {x[fin][bad][:5]} vs {y[fin][bad][:5]}"


def sorted_rows(batch: pa.RecordBatch, key_cols):
    rows = list(zip(*(batch.column(i).to_pylist() for i in range(batch.num_columns))))
    return sorted(rows, key=lambda r: tuple((v is None, v) for v in (r[k] for k in key_cols)))
