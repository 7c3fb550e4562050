"""GPU hash aggregation parity against the CPU oracle (hash_aggregate.rs)."""
import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from golden import reference_kat as K
from helpers import assert_batches_equal, close
from prism_gpu import AggExpr, AggFunc, HashAggConfig

pytestmark = pytest.mark.gpu

C1_AGGS = [
    AggExpr(1, AggFunc.Count, "cnt"),
    AggExpr(1, AggFunc.Sum, "sum_v_i"),
    AggExpr(1, AggFunc.Min, "min_v_i"),
    AggExpr(1, AggFunc.Max, "max_v_i"),
    AggExpr(2, AggFunc.Sum, "sum_v_f"),
    AggExpr(2, AggFunc.Avg, "avg_v_f"),
]


def c1_batch(n, seed=0, groups=1024):
    rng = np.random.default_rng(seed)
    return pa.RecordBatch.from_arrays(
        [pa.array(rng.integers(0, groups, n)), pa.array(rng.integers(-1_000_000, 1_000_001, n)), pa.array(rng.random(n))],
        names=["g", "v_i", "v_f"],
    )


def test_reference_known_answers(ctx):
    out = prism_gpu.hash_aggregate(K.sales_batch(), K.SUM_BY_REGION)
    assert out.num_rows == 2 and sum(out.column(1).to_pylist()) == 800.0
    assert_batches_equal(out, oracle.hash_aggregate(K.sales_batch(), K.SUM_BY_REGION))
    assert_batches_equal(prism_gpu.hash_aggregate(K.sales_batch(), K.COUNT_AND_AVG), oracle.hash_aggregate(K.sales_batch(), K.COUNT_AND_AVG))
    out = prism_gpu.hash_aggregate(K.large_int64_batch(), K.GLOBAL_COUNT_DISTINCT)
    assert out.column(0).to_pylist() == [2]
    out = prism_gpu.hash_aggregate(K.labels_batch(), K.GROUPED_COUNT_DISTINCT)
    assert dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist())) == {"east": 2, "west": 2}


def test_partial_merge_known_answer(ctx):
    merged = prism_gpu.hash_aggregate_batches(K.partial_batches(), K.MERGE_CONFIG)
    assert_batches_equal(merged, oracle.hash_aggregate_batches(K.partial_batches(), K.MERGE_CONFIG))


@pytest.mark.parametrize("n", [1, 31, 1000, 100_000, 1_000_000])
def test_c1_shape_bit_exact(ctx, n):
    b = c1_batch(n, seed=n)
    cfg = HashAggConfig([0], C1_AGGS)
    got = prism_gpu.hash_aggregate(b, cfg)
    ref = oracle.hash_aggregate(b, cfg)
    # integer aggregates are bit-exact; the Float64 sum/avg within 1e-12
    assert_batches_equal(got, ref, float_cols=(5, 6))
    # and the Float64 SUM is the correctly rounded exact sum
    g = b.column(0).to_numpy()
    f = b.column(2).to_numpy()
    keys = got.column(0).to_numpy()
    exact = [oracle.exact_sum_f64(f[g == k]) for k in keys[:50]]
    assert np.array_equal(got.column(5).to_numpy()[:50], np.array(exact))


@pytest.mark.parametrize("groups", [1, 7, 5000, 200_000])
def test_cardinalities(ctx, groups):
    b = c1_batch(300_000, seed=groups, groups=groups)
    cfg = HashAggConfig([0], C1_AGGS)
    assert_batches_equal(prism_gpu.hash_aggregate(b, cfg), oracle.hash_aggregate(b, cfg), float_cols=(5, 6))


def test_multi_batch_first_seen_order(ctx):
    bs = [c1_batch(50_000, seed=s, groups=3000) for s in range(5)] + [c1_batch(10, seed=9).slice(0, 0)]
    cfg = HashAggConfig([0], C1_AGGS)
    assert_batches_equal(prism_gpu.hash_aggregate_batches(bs, cfg), oracle.hash_aggregate_batches(bs, cfg, n_threads=4), float_cols=(5, 6))


def test_null_keys_share_group_with_zero(ctx):
    b = pa.RecordBatch.from_arrays([pa.array([0, None, 1, None, 5], pa.int64()), pa.array([1.0, 2.0, 3.0, 4.0, 5.0])], names=["g", "v"])
    cfg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Count, "c")])
    assert_batches_equal(prism_gpu.hash_aggregate(b, cfg), oracle.hash_aggregate(b, cfg))


def test_sentinel_key_values(ctx):
    ks = np.array([-1, 0, np.iinfo(np.int64).min, np.iinfo(np.int64).max, -1, 3], dtype=np.int64)
    b = pa.RecordBatch.from_arrays([pa.array(ks), pa.array(np.arange(6, dtype=np.int64))], names=["g", "v"])
    cfg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Max, "m")])
    assert_batches_equal(prism_gpu.hash_aggregate(b, cfg), oracle.hash_aggregate(b, cfg))


def test_string_and_multi_keys(ctx):
    rng = np.random.default_rng(5)
    n = 60_000
    regions = np.array(["east", "west", "north", "south", "", "a-much-longer-region-name"])
    b = pa.RecordBatch.from_arrays(
        [pa.array(regions[rng.integers(0, 6, n)]), pa.array(rng.integers(0, 50, n).astype(np.int32)), pa.array(rng.standard_normal(n) * 1e6)],
        names=["r", "k", "v"],
    )
    for gb in ([0], [1], [0, 1], [1, 0]):
        cfg = HashAggConfig(gb, [AggExpr(2, AggFunc.Sum, "s"), AggExpr(2, AggFunc.Min, "mn"), AggExpr(2, AggFunc.Avg, "a"), AggExpr(1, AggFunc.CountDistinct, "d")])
        nkeys = len(gb)
        assert_batches_equal(prism_gpu.hash_aggregate(b, cfg), oracle.hash_aggregate(b, cfg), float_cols=(nkeys, nkeys + 2))


def test_dictionary_keys_dense_path(ctx):
    rng = np.random.default_rng(8)
    n = 200_000
    flag = pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 3, n).astype(np.int8)), pa.array(["A", "N", "R"]))
    status = pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 2, n).astype(np.int8)), pa.array(["F", "O"]))
    b = pa.RecordBatch.from_arrays([flag, status, pa.array(rng.integers(0, 10**9, n))], names=["flag", "status", "v"])
    cfg = HashAggConfig([0, 1], [AggExpr(2, AggFunc.Sum, "s"), AggExpr(2, AggFunc.Count, "c"), AggExpr(2, AggFunc.Avg, "a")])
    assert_batches_equal(prism_gpu.hash_aggregate(b, cfg), oracle.hash_aggregate(b, cfg), float_cols=(4,))


def test_global_aggregates_skip_nulls(ctx):
    rng = np.random.default_rng(2)
    v = rng.standard_normal(100_000)
    mask = rng.random(100_000) < 0.1
    b = pa.RecordBatch.from_arrays([pa.array(v, mask=mask), pa.array(rng.integers(0, 100, 100_000), mask=mask)], names=["f", "i"])
    cfg = HashAggConfig(
        [],
        [
            AggExpr(0, AggFunc.Sum, "s"),
            AggExpr(0, AggFunc.Count, "c"),
            AggExpr(0, AggFunc.Avg, "a"),
            AggExpr(0, AggFunc.Min, "mn"),
            AggExpr(0, AggFunc.Max, "mx"),
            AggExpr(1, AggFunc.CountDistinct, "d"),
            AggExpr(1, AggFunc.Sum, "si"),
        ],
    )
    assert_batches_equal(prism_gpu.hash_aggregate(b, cfg), oracle.hash_aggregate(b, cfg), float_cols=(0, 2, 6))


def test_float_specials_and_wide_range(ctx):
    vals = [1e300, -1e300, 1e-300, 3.5, float("inf"), 2.0, float("nan"), -0.0, 1e20, -1e20, 7.0]
    g = [0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 4]
    b = pa.RecordBatch.from_arrays([pa.array(g, pa.int64()), pa.array(vals)], names=["g", "v"])
    cfg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Min, "mn"), AggExpr(1, AggFunc.Max, "mx"), AggExpr(1, AggFunc.Count, "c")])
    got = prism_gpu.hash_aggregate(b, cfg)
    ref = oracle.hash_aggregate(b, cfg)
    assert_batches_equal(got, ref, float_cols=(1,))


def test_empty_inputs(ctx):
    b = c1_batch(10).slice(0, 0)
    cfg = HashAggConfig([0], C1_AGGS)
    assert_batches_equal(prism_gpu.hash_aggregate(b, cfg), oracle.hash_aggregate(b, cfg))


def test_unsupported_aggregate_input(ctx):
    with pytest.raises(prism_gpu.PrismError) as e:
        prism_gpu.hash_aggregate(K.sales_batch(), HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "x")]))
    assert e.value.kind == "UnsupportedAggregation"


def test_deterministic_across_runs(ctx):
    b = c1_batch(500_000, seed=77)
    cfg = HashAggConfig([0], C1_AGGS)
    first = prism_gpu.hash_aggregate(b, cfg)
    for _ in range(3):
        assert prism_gpu.hash_aggregate(b, cfg).equals(first)


@pytest.mark.parametrize("scale", [1e-40, 1e-30, 3e-39])
def test_float_sums_below_the_window_bottom(ctx, scale):
    """Groups whose values all lie near or below 2^-128 (no large value in the
    call): every mantissa bit counts, so SUM / AVG stay within 1e-12 of the
    reference's sequential sums (and equal the correctly rounded exact sum)."""
    rng = np.random.default_rng(int(-np.log10(scale)))
    n = 20_000
    g = rng.integers(0, 13, n)
    v = rng.random(n) * scale
    b = pa.RecordBatch.from_arrays([pa.array(g), pa.array(v)], names=["g", "v"])
    cfg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Avg, "a"), AggExpr(1, AggFunc.Count, "c")])
    got = prism_gpu.hash_aggregate(b, cfg)
    assert_batches_equal(got, oracle.hash_aggregate(b, cfg), float_cols=(1, 2))
    keys = got.column(0).to_numpy()
    exact = np.array([oracle.exact_sum_f64(v[g == k]) for k in keys])
    assert np.array_equal(got.column(1).to_numpy(), exact)
    # the same values under a dictionary key (few dense groups) and globally
    d = pa.DictionaryArray.from_arrays(pa.array((g % 3).astype(np.int8)), pa.array(["x", "y", "z"]))
    bd = pa.RecordBatch.from_arrays([d, pa.array(v)], names=["d", "v"])
    assert_batches_equal(prism_gpu.hash_aggregate(bd, cfg), oracle.hash_aggregate(bd, cfg), float_cols=(1, 2))
    gcfg = HashAggConfig([], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Avg, "a")])
    assert_batches_equal(prism_gpu.hash_aggregate(b, gcfg), oracle.hash_aggregate(b, gcfg), float_cols=(0, 1))


def test_float_sum_mixed_tiny_and_unit_values(ctx):
    """A value near 1e-30 beside values near 1: the sum keeps the tiny value's
    contribution exactly as the correctly rounded sum does."""
    v = np.array([1e-30, 1.0, 2.5e-31, 0.75, 1e-40, 3.0], dtype=np.float64)
    g = np.array([0, 0, 1, 1, 2, 2], dtype=np.int64)
    b = pa.RecordBatch.from_arrays([pa.array(g), pa.array(v)], names=["g", "v"])
    cfg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s")])
    got = prism_gpu.hash_aggregate(b, cfg)
    assert_batches_equal(got, oracle.hash_aggregate(b, cfg), float_cols=(1,))
    exact = np.array([oracle.exact_sum_f64(v[g == k]) for k in got.column(0).to_numpy()])
    assert np.array_equal(got.column(1).to_numpy(), exact)


def test_generated_kernels_reused_per_plan(ctx):
    """The generated aggregation kernels are looked up by plan, not by their
    regenerated source: plans that differ only in a key column's type, its
    nulls, the row count or the aggregate list, interleaved and each run
    twice in one process, all equal the oracle."""
    rng = np.random.default_rng(404)

    def batch(n, key_type, nulls):
        k = rng.integers(0, 3000, n)
        mask = (rng.random(n) < 0.05) if nulls else None
        return pa.RecordBatch.from_arrays(
            [pa.array(k.astype(key_type), mask=mask), pa.array(rng.integers(-1000, 1000, n)), pa.array(rng.random(n))],
            names=["k", "v", "f"])

    cfgs = [HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(2, AggFunc.Max, "m")]),
            HashAggConfig([0], [AggExpr(2, AggFunc.Sum, "sf"), AggExpr(1, AggFunc.Count, "n"), AggExpr(1, AggFunc.Min, "mn")])]
    batches = [batch(50_000, np.int64, False), batch(50_000, np.int32, False), batch(50_000, np.int64, True),
               batch(70_001, np.int64, False)]
    for _ in range(2):
        for b in batches:
            for cfg in cfgs:
                got = prism_gpu.hash_aggregate(b, cfg)
                ref = oracle.hash_aggregate(b, cfg)
                assert_batches_equal(got, ref, float_cols=tuple(i for i in range(ref.num_columns)
                                                                 if pa.types.is_floating(ref.schema.field(i).type)))
