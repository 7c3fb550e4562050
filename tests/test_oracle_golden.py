"""Pins the CPU oracle to the reference's own known-answer tests.

Every case in tests/golden/reference_kat.py comes from a reference unit test
(file:line cited there); the oracle must reproduce what the reference asserts
before it is trusted as the parity checker for the GPU path.
"""
import math

import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
from golden import reference_kat as K
from prism_gpu.config import AggExpr, AggFunc, HashAggConfig, HashJoinConfig, JoinType, Predicate, ScalarValue


@pytest.mark.parametrize("name,jt,rows,cols", K.JOIN_CASES)
def test_join_known_answers(name, jt, rows, cols):
    out = oracle.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(jt))
    assert out.num_rows == rows
    if cols is not None:
        assert out.num_columns == cols


def test_inner_join_values_and_right_suffix():
    out = oracle.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(JoinType.Inner))
    assert out.schema.names == ["emp_id", "name", "dept_id", "dept_id_right", "dept_name"]
    assert out.column(0).to_pylist() == [100, 101, 102]
    assert out.column(4).to_pylist() == ["Engineering", "Sales", "Engineering"]


def test_sum_by_region():
    out = oracle.hash_aggregate(K.sales_batch(), K.SUM_BY_REGION)
    assert out.num_rows == 2 and out.num_columns == 2
    assert sum(out.column(1).to_pylist()) == 800.0
    # first-seen order (east first), as hash_aggregate.rs:302-314 emits it
    assert out.column(0).to_pylist() == ["east", "west"]
    assert out.column(1).to_pylist() == [300.0, 500.0]


def test_count_and_avg():
    out = oracle.hash_aggregate(K.sales_batch(), K.COUNT_AND_AVG)
    assert out.num_rows == 2 and out.num_columns == 3
    assert out.schema.field(1).type == pa.int64()
    assert out.column(1).to_pylist() == [3, 2]
    assert out.column(2).to_pylist() == [100.0, 250.0]


def test_global_count_distinct_large_int64():
    out = oracle.hash_aggregate(K.large_int64_batch(), K.GLOBAL_COUNT_DISTINCT)
    assert out.column(0).to_pylist() == [2]


def test_grouped_count_distinct_utf8():
    out = oracle.hash_aggregate(K.labels_batch(), K.GROUPED_COUNT_DISTINCT)
    got = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert got == {"east": 2, "west": 2}


def test_filter_gt():
    b = K.fp_test_batch()
    mask = oracle.evaluate_predicate(b, K.FILTER_GT)
    out = oracle.filter_batch(b, mask)
    assert out.column(0).to_pylist() == [4, 5]


def test_filter_and_project():
    out = oracle.filter_and_project(K.fp_test_batch(), K.FILTER_LE, [1, 2])
    assert out.num_rows == 3 and out.num_columns == 2
    names = out.column(0).to_pylist()
    assert names[0] == "alice" and names[2] == "carol"


def test_compound_predicate():
    b = K.fp_test_batch()
    out = oracle.filter_batch(b, oracle.evaluate_predicate(b, K.COMPOUND))
    assert out.num_rows == 3


def test_predicate_literal_broadcasts():
    b = K.fp_test_batch()
    mask = oracle.evaluate_predicate(b, Predicate.Literal(True))
    assert len(mask) == b.num_rows and all(v is True for v in mask.to_pylist())


def test_if_then_projects_string_branches():
    out = oracle.project_batch_with_exprs(K.if_then_batch(), [0], [K.IF_THEN_EXPR])
    assert out.column(1).to_pylist() == ["owner", "b", "c"]
    assert out.schema.names == ["id", "expr_0"]


def test_fused_join_aggregate():
    out = oracle.join_aggregate(K.fused_left_batches(), K.fused_right_batch(), [0], [0], K.FUSED_PROJECT_COLS, K.FUSED_EXPRS, K.FUSED_AGG)
    rows = {s: (v, c) for s, v, c in zip(*(out.column(i).to_pylist() for i in range(3)))}
    assert rows == K.FUSED_EXPECTED


def test_fused_join_avg():
    out = oracle.join_aggregate(K.fused_avg_left(), K.fused_right_batch(), [0], [0], K.FUSED_AVG_COLS, [], K.FUSED_AVG_AGG)
    rows = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert rows == K.FUSED_AVG_EXPECTED


def test_distributed_partial_merge():
    merged = oracle.hash_aggregate_batches(K.partial_batches(), K.MERGE_CONFIG)
    # reconstruct_original_aggregate_batch (executor.rs:745-812): SUM, COUNT, AVG=sum/count
    st = merged.column(0).to_pylist()
    s, c, s2, c2 = (merged.column(i).to_pylist() for i in range(1, 5))
    rows = {st[i]: (s[i], int(c[i]), s2[i] / c2[i] if c2[i] > 0 else 0.0) for i in range(len(st))}
    assert rows == K.MERGE_EXPECTED


def test_reducer_merge_reconstructs_original_aggregates():
    """handler.rs:1378-1460 through the oracle's restatement of the whole
    reducer (final merge config, hash aggregation, reconstruct)."""
    out = oracle.merge_partial_aggregates(K.partial_batches(), K.MERGE_ORIGINAL)
    assert out.schema.types == [pa.utf8(), pa.float64(), pa.int64(), pa.float64()]
    rows = {r["status"]: (r["agg_0"], r["agg_1"], r["agg_2"]) for r in out.to_pylist()}
    assert rows == K.MERGE_EXPECTED


def test_worker_aggregate_expansion_matches_oracle():
    """prism_expand_worker_aggregates (host-only C entry point) against the
    oracle's restatement of expand_worker_aggregates (handler.rs:397-428)."""
    import prism_gpu
    from prism_gpu import AggExpr, AggFunc, HashAggConfig

    F = AggFunc
    cfg = HashAggConfig([2, 0], [AggExpr(1, F.Avg, "a"), AggExpr(3, F.Min, "b"), AggExpr(1, F.CountDistinct, "c"),
                                 AggExpr(4, F.Avg, "d"), AggExpr(0, F.Count, "e"), AggExpr(5, F.Max, "f")])
    got = prism_gpu.expand_worker_aggregates(cfg)
    ref, mapping = oracle.expand_worker_aggregates(cfg)
    assert got == ref
    assert mapping == [[0, 1], [2], [3], [4, 5], [6], [7]]
    assert [a.output_name for a in got.aggregates] == [f"agg_{i}" for i in range(8)]
    assert prism_gpu.expand_worker_aggregates(K.MERGE_ORIGINAL).aggregates == [
        AggExpr(1, F.Sum, "agg_0"), AggExpr(1, F.Count, "agg_1"), AggExpr(1, F.Sum, "agg_2"), AggExpr(1, F.Count, "agg_3")]


def test_like_pipeline_count():
    # native/prism-executor/tests/integration.rs:302-340: '%coast%' matches 40,000 of 100K
    regions = ["east_coast", "west_coast", "central", "north_west", "south_east"]
    n = 100_000
    b = pa.RecordBatch.from_arrays([pa.array(np.arange(n, dtype=np.int64)), pa.array([regions[i % 5] for i in range(n)])], names=["id", "region"])
    mask = oracle.evaluate_predicate(b, Predicate.Like(1, "%coast%"))
    assert mask.to_numpy(zero_copy_only=False).sum() == 40_000


def test_q1_like_group_count():
    # integration.rs:158-213: aggregate lineitem by shipregion -> 5 rows
    n = 100_000
    regions = ["EAST", "WEST", "NORTH", "SOUTH", "CENTRAL"]
    i = np.arange(n)
    b = pa.RecordBatch.from_arrays(
        [pa.array(i.astype(np.int64)), pa.array((i % 50 + 1).astype(np.float64)), pa.array((i % 10000) * 1.23 + 10.0), pa.array([regions[k % 5] for k in range(n)])],
        names=["orderkey", "quantity", "extendedprice", "shipregion"],
    )
    cfg = HashAggConfig([3], [AggExpr(1, AggFunc.Sum, "sum_qty"), AggExpr(2, AggFunc.Sum, "sum_price"), AggExpr(0, AggFunc.Count, "cnt")])
    out = oracle.hash_aggregate(b, cfg)
    assert out.num_rows == 5
    assert out.column(3).to_pylist() == [20_000] * 5


# ---- oracle vs an independent implementation (pyarrow Acero) -------------


def test_oracle_join_matches_acero():
    rng = np.random.default_rng(7)
    build = pa.table({"k": rng.permutation(5000).astype(np.int64), "p": rng.integers(0, 1 << 40, 5000)})
    probe = pa.table({"k": rng.integers(0, 6000, 20000).astype(np.int64), "x": rng.integers(0, 100, 20000).astype(np.int32)})
    pb, bb = probe.to_batches()[0], build.to_batches()[0]
    out = oracle.hash_join(pb, bb, HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0]))
    ac = probe.join(build, "k", join_type="inner")
    mine = sorted(zip(out.column(0).to_pylist(), out.column(1).to_pylist(), out.column(3).to_pylist()))
    theirs = sorted(zip(ac.column("k").to_pylist(), ac.column("x").to_pylist(), ac.column("p").to_pylist()))
    assert mine == theirs


def test_oracle_groupby_matches_acero():
    rng = np.random.default_rng(11)
    n = 50_000
    t = pa.table({"g": rng.integers(0, 300, n), "v": rng.integers(-1000, 1000, n), "f": rng.random(n)})
    cfg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Min, "mn"), AggExpr(1, AggFunc.Max, "mx"), AggExpr(2, AggFunc.Count, "c")])
    out = oracle.hash_aggregate(t.to_batches()[0], cfg)
    ac = t.group_by("g").aggregate([("v", "sum"), ("v", "min"), ("v", "max"), ("f", "count")])
    mine = {g: (s, mn, mx, c) for g, s, mn, mx, c in zip(*(out.column(i).to_pylist() for i in range(5)))}
    theirs = {g: (float(s), float(mn), float(mx), c) for g, s, mn, mx, c in zip(*(ac.column(n).to_pylist() for n in ["g", "v_sum", "v_min", "v_max", "f_count"]))}
    assert mine == theirs


def test_exact_sum_is_correctly_rounded():
    vals = [1e16, 1.0, -1e16, 3.0, 2.0 ** -60]
    assert oracle.exact_sum_f64(vals) == 4.0 + 2.0 ** -60
    assert oracle.exact_sum_f64([0.1] * 10) == math.fsum([0.1] * 10)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(100_000) * 10.0 ** rng.integers(-20, 20, 100_000)
    assert oracle.exact_sum_f64(x) == math.fsum(x)


def test_first_seen_order_over_batches():
    # first-seen order over the concatenated batches survives the chunked merge
    b1 = pa.RecordBatch.from_arrays([pa.array([5, 3, 5], pa.int64()), pa.array([1.0, 2.0, 3.0])], names=["g", "v"])
    b2 = pa.RecordBatch.from_arrays([pa.array([7, 3, 9], pa.int64()), pa.array([4.0, 5.0, 6.0])], names=["g", "v"])
    for threads in (1, 2, 4):
        out = oracle.hash_aggregate_batches([b1, b2], HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s")]), n_threads=threads)
        assert out.column(0).to_pylist() == [5, 3, 7, 9]
        assert out.column(1).to_pylist() == [4.0, 7.0, 4.0, 6.0]


def test_null_key_collides_with_zero_in_grouped_path():
    # FxHash: a null key writes 0u8 -> write_u64(0), the same as key 0
    # (hash_aggregate.rs:492-497), so null and 0 share one group.
    b = pa.RecordBatch.from_arrays([pa.array([0, None, 1], pa.int64()), pa.array([1.0, 2.0, 3.0])], names=["g", "v"])
    out = oracle.hash_aggregate(b, HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s")]))
    assert out.column(0).to_pylist() == [0, 1]
    assert out.column(1).to_pylist() == [3.0, 3.0]


def test_left_join_unmatched_rows_take_build_row_zero():
    # left_join_indices pushes build index 0 for unmatched probe rows
    # (hash_join.rs:472-477), so they carry build row 0's values.
    out = oracle.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(JoinType.Left))
    assert out.num_rows == 4
    assert out.column(0).to_pylist() == [100, 101, 102, 103]
    assert out.column(4).to_pylist() == ["Engineering", "Sales", "Engineering", "Engineering"]


def test_errors_mirror_prism_error():
    b = K.fp_test_batch()
    with pytest.raises(oracle.OracleError) as e:
        oracle.evaluate_predicate(b, Predicate.Eq(0, ScalarValue.Float64(1.0)))  # Int64 vs Float64
    assert e.value.kind == "InvalidArgument"
