"""Parquet inputs for the scan tests, written with pyarrow at test time.

`reference_test_file` restates the file of parquet_scan.rs's own tests
(build_test_parquet_bytes, parquet_scan.rs:557-599): 500 rows of
id Int64 = 0..499, value Float64 = id, name Utf8 = alpha / beta / gamma /
delta / epsilon in runs of 100, SNAPPY, 100-row row groups with chunk
statistics. `typed_table` is a seeded table with every type the GPU decoder
reads, with nulls.
"""
import os

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq

NAMES = ["alpha", "beta", "gamma", "delta", "epsilon"]


def reference_test_table() -> pa.Table:
    ids = np.arange(500, dtype=np.int64)
    schema = pa.schema([pa.field("id", pa.int64(), False), pa.field("value", pa.float64(), False),
                        pa.field("name", pa.utf8(), False)])
    return pa.table([pa.array(ids), pa.array(ids.astype(np.float64)), pa.array([NAMES[i // 100] for i in range(500)])],
                    schema=schema)


def reference_test_file(directory: str, row_group_size: int = 100) -> str:
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, "test.parquet")
    pq.write_table(reference_test_table(), path, compression="snappy", row_group_size=row_group_size,
                   write_statistics=True)
    return path


def typed_table(n: int, seed: int, nulls: bool = True) -> pa.Table:
    rng = np.random.default_rng(seed)

    def mask(p):
        return (rng.random(n) < p) if nulls else None

    words = np.array(["", "a", "bb", "ccc", "delta", "epsilon-" * 3, "z" * 40, "été", "日本"])
    many = np.array([f"key-{i:07d}" for i in range(max(1, n // 3))])
    return pa.table({
        "i32": pa.array(rng.integers(-2**31, 2**31 - 1, n).astype(np.int32), mask=mask(0.1)),
        "i64": pa.array(rng.integers(-2**62, 2**62, n), mask=mask(0.05)),
        "f32": pa.array(rng.normal(0, 1e3, n).astype(np.float32), mask=mask(0.1)),
        "f64": pa.array(rng.normal(0, 1e6, n), mask=mask(0.1)),
        "flag": pa.array(rng.random(n) < 0.3, mask=mask(0.1)),
        "day": pa.array(rng.integers(0, 20000, n).astype(np.int32), type=pa.date32(), mask=mask(0.1)),
        "word": pa.array(words[rng.integers(0, len(words), n)], mask=mask(0.1)),
        "key": pa.array(many[rng.integers(0, len(many), n)], mask=mask(0.02)),
        "small": pa.array(rng.integers(0, 4, n), mask=mask(0.5)),
        "dense": pa.array(np.arange(n, dtype=np.int64)),
    })
