"""GPU sort / top-N (prism_sort_batch, the radix sort) against the oracle's
restatement of sort.rs: every key type, both directions and null placements,
several keys, limits, ties (stable), sizes spanning many tiles, and the
reference's own known answers."""
import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from golden import reference_kat as K
from helpers import assert_batches_equal
from prism_gpu import NullOrdering as N
from prism_gpu import SortDirection as D
from prism_gpu import SortKey

pytestmark = pytest.mark.gpu


def table(n, seed, nulls=True):
    rng = np.random.default_rng(seed)

    def mask(p):
        return (rng.random(n) < p) if nulls else None

    f = rng.normal(0, 100, n).round(2)
    f[rng.random(n) < 0.02] = np.nan
    f[rng.random(n) < 0.02] = -np.nan
    f[rng.random(n) < 0.02] = -0.0
    f[rng.random(n) < 0.02] = 0.0
    f[rng.random(n) < 0.01] = np.inf
    f[rng.random(n) < 0.01] = -np.inf
    words = np.array(["", "a", "a\x00", "ab", "abc", "b", "ba", "zz" * 9, "zz" * 9 + "a", "\xff"])
    dec = [None if (nulls and rng.random() < 0.05) else int(v) for v in rng.integers(-10**15, 10**15, n)]
    return pa.RecordBatch.from_arrays(
        [pa.array(rng.integers(-50, 50, n), mask=mask(0.05)),
         pa.array(f, mask=mask(0.05)),
         pa.array(words[rng.integers(0, len(words), n)], mask=mask(0.05)),
         pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 4, n).astype(np.int8), mask=mask(0.05)),
                                        pa.array(["pear", "apple", "fig", "apple pie"])),
         pa.array(rng.integers(-3, 3, n).astype(np.int32), mask=mask(0.05)),
         pa.array(rng.random(n) < 0.5, mask=mask(0.05)),
         pa.array(rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True), mask=mask(0.05)),
         pa.array(rng.normal(0, 1, n).astype(np.float32), mask=mask(0.05)),
         pa.array(rng.integers(0, 20000, n).astype(np.int32), type=pa.date32()),
         pa.array([None if d is None else d for d in dec], type=pa.decimal128(20, 2)),
         pa.array(np.arange(n))],
        names=["i", "f", "s", "d", "i32", "b", "u64", "f32", "day", "dec", "row"])


SPECS = {
    "int_asc": [(0, D.Asc)],
    "float_desc": [(1, D.Desc)],
    "utf8_asc": [(2, D.Asc)],
    "dict_desc": [(3, D.Desc)],
    "int32_float": [(4, D.Desc), (1, D.Asc)],
    "bool_utf8_int": [(5, D.Asc), (2, D.Desc), (0, D.Asc)],
    "u64_desc": [(6, D.Desc)],
    "f32_asc": [(7, D.Asc)],
    "date_dec": [(8, D.Desc), (9, D.Asc)],
    "dec_desc": [(9, D.Desc)],
}


@pytest.mark.parametrize("nulls", [N.NullsFirst, N.NullsLast])
@pytest.mark.parametrize("spec", sorted(SPECS))
def test_sort_matches_oracle(ctx, spec, nulls):
    b = table(20_000, 5)
    keys = [SortKey(c, d, nulls) for c, d in SPECS[spec]]
    got = prism_gpu.sort_batch(b, keys, ctx=ctx)
    ref = oracle.sort_batch(b, keys)
    assert got.column(10).equals(ref.column(10)), "row order differs"
    assert_batches_equal(got, ref, float_cols=(1, 7))


@pytest.mark.parametrize("limit", [0, 1, 7, 4096, 50_000])
def test_top_n(ctx, limit):
    """sort_batch_limit / topn_single_col: the first `limit` rows of the sort."""
    b = table(30_000, 9)
    keys = [SortKey(1, D.Desc, N.NullsLast)]
    got = prism_gpu.sort_batch(b, keys, limit=limit, ctx=ctx)
    ref = oracle.sort_batch(b, keys, limit=limit)
    assert got.num_rows == ref.num_rows == min(limit, b.num_rows)
    assert got.column(10).equals(ref.column(10))


def test_many_tiles_and_ties(ctx):
    """3M rows (hundreds of tiles per pass), heavy ties on the first key:
    the order among ties is the input order."""
    rng = np.random.default_rng(1)
    n = 3_000_000
    b = pa.RecordBatch.from_arrays([pa.array(rng.integers(0, 100, n)), pa.array(rng.normal(0, 1, n)),
                                    pa.array(np.arange(n))], names=["k", "x", "row"])
    keys = [SortKey(0, D.Asc, N.NullsLast)]
    got = prism_gpu.sort_batch(b, keys, ctx=ctx)
    ref = oracle.sort_batch(b, keys)
    assert got.column(2).equals(ref.column(2))
    keys2 = [SortKey(0, D.Desc, N.NullsFirst), SortKey(1, D.Asc, N.NullsLast)]
    got2 = prism_gpu.sort_batch(b, keys2, limit=1000, ctx=ctx)
    ref2 = oracle.sort_batch(b, keys2, limit=1000)
    assert got2.column(2).equals(ref2.column(2))


def test_edges(ctx):
    b = table(100, 3)
    assert prism_gpu.sort_batch(b, [], ctx=ctx).column(10).equals(b.column(10))
    assert prism_gpu.sort_batch(b.slice(0, 0), [SortKey(0)], ctx=ctx).num_rows == 0
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.sort_batch(b, [SortKey(42)], ctx=ctx)


def test_reference_known_answers(ctx):
    """sort.rs's own tests (sort.rs:255-299)."""
    b = K.sort_test_batch()
    names = prism_gpu.sort_batch(b, K.SORT_BY_NAME_ASC, ctx=ctx).column(0).to_pylist()
    assert names[0] == "Alice" and names[4] == "Eve"
    top = prism_gpu.sort_batch(b, K.SORT_BY_SCORE_DESC, limit=3, ctx=ctx)
    assert top.num_rows == 3 and top.column(2)[0].as_py() == 92.0
    multi = prism_gpu.sort_batch(b, K.SORT_MULTI_KEY, ctx=ctx)
    assert multi.column(1)[0].as_py() == 25 and multi.column(2)[0].as_py() == 92.0


@pytest.mark.parametrize("kind", ["f64", "i32_nulls", "u8_nulls", "f32_desc_nulls_first", "bool", "i64_ties"])
@pytest.mark.parametrize("limit", [0, 1, 100, 5000])
def test_top_n_select(ctx, kind, limit):
    """Top-N of one fixed-width key over 1.5M rows: the radix-select path
    (rows narrowed before the sort) gives the oracle's rows, ties included."""
    rng = np.random.default_rng(sum(map(ord, kind)))
    n = 1_500_000
    if kind == "f64":
        col, key = pa.array(rng.normal(0, 1, n)), SortKey(0, D.Desc, N.NullsLast)
    elif kind == "i32_nulls":
        col, key = pa.array(rng.integers(-1000, 1000, n).astype(np.int32), mask=rng.random(n) < 0.2), SortKey(0, D.Asc, N.NullsFirst)
    elif kind == "u8_nulls":
        col, key = pa.array(rng.integers(0, 256, n).astype(np.uint8), mask=rng.random(n) < 0.01), SortKey(0, D.Desc, N.NullsLast)
    elif kind == "f32_desc_nulls_first":
        col, key = pa.array(rng.normal(0, 1, n).astype(np.float32), mask=rng.random(n) < 0.001), SortKey(0, D.Desc, N.NullsFirst)
    elif kind == "bool":
        col, key = pa.array(rng.random(n) < 0.001), SortKey(0, D.Desc, N.NullsLast)
    else:
        col, key = pa.array(rng.integers(0, 3, n)), SortKey(0, D.Asc, N.NullsLast)
    b = pa.RecordBatch.from_arrays([col, pa.array(np.arange(n))], names=["k", "row"])
    got = prism_gpu.sort_batch(b, [key], limit=limit, ctx=ctx)
    ref = oracle.sort_batch(b, [key], limit=limit)
    assert got.num_rows == ref.num_rows == limit
    assert got.column(1).equals(ref.column(1))
