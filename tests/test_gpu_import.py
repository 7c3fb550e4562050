"""Import of pageable host Arrow buffers through page-locked staging: large
columns (several staging chunks, sliced inputs, nulls, Utf8) arrive intact,
and pinned inputs keep the direct path."""
import numpy as np
import pyarrow as pa
import pytest

import prism_gpu

pytestmark = pytest.mark.gpu


def test_pageable_import_round_trip(ctx):
    rng = np.random.default_rng(3)
    n = 12_000_000  # 96 MB per Int64 column: three 32 MB staging chunks each
    words = pa.array(["", "ab", "staging", "z" * 33])
    b = pa.RecordBatch.from_arrays([
        pa.array(rng.integers(-2**62, 2**62, n)),
        pa.array(rng.random(n), mask=rng.random(n) < 0.1),
        words.take(pa.array(rng.integers(0, 4, n))),
        pa.array(rng.integers(0, 2**31 - 1, n).astype(np.int32)),
    ], names=["a", "b", "s", "c"])
    for sl in (b, b.slice(1_234_567, 7_000_001)):
        d = prism_gpu.DeviceBatch.from_arrow(sl, ctx)
        assert d.to_arrow().equals(sl)
        d.free()


def test_pinned_import_direct(ctx):
    import torch

    n = 4_000_000
    t = torch.arange(n, dtype=torch.int64).pin_memory()
    arr = pa.foreign_buffer(t.data_ptr(), n * 8, base=t)
    b = pa.RecordBatch.from_arrays([pa.Array.from_buffers(pa.int64(), n, [None, arr])], names=["x"])
    d = prism_gpu.DeviceBatch.from_arrow(b, ctx)
    assert d.to_arrow().column(0).equals(b.column(0))
