"""Known-answer cases transcribed from the reference's own unit tests.

Each case builds the same input batches as the cited reference test and
records the result the reference asserts. The GPU path and the CPU oracle are
both checked against them (tests/test_oracle_golden.py for the oracle;
tests/test_gpu_join.py, test_gpu_agg.py, test_gpu_filter_project.py,
test_gpu_fused.py, test_gpu_sort.py and test_gpu_distributed.py on the GPU).
No values here are invented: where the reference asserts only a shape (row or
column count) the case asserts only that shape.
"""
from __future__ import annotations

import pyarrow as pa

from prism_gpu.config import (
    AggExpr,
    NullOrdering,
    SortDirection,
    SortKey,
    AggFunc,
    ArithmeticOp,
    HashAggConfig,
    HashJoinConfig,
    JoinType,
    Predicate,
    ScalarExpr,
    ScalarValue,
)


# ---------------------------------------------------------------- join -----
# native/prism-executor/src/hash_join.rs:678-708
def join_build_side() -> pa.RecordBatch:
    return pa.RecordBatch.from_arrays(
        [pa.array([1, 2, 3], pa.int64()), pa.array(["Engineering", "Sales", "Marketing"], pa.utf8())],
        schema=pa.schema([pa.field("dept_id", pa.int64(), False), pa.field("dept_name", pa.utf8(), False)]),
    )


def join_probe_side() -> pa.RecordBatch:
    return pa.RecordBatch.from_arrays(
        [
            pa.array([100, 101, 102, 103], pa.int64()),
            pa.array(["Alice", "Bob", "Carol", "Dave"], pa.utf8()),
            pa.array([1, 2, 1, 99], pa.int64()),
        ],
        schema=pa.schema(
            [pa.field("emp_id", pa.int64(), False), pa.field("name", pa.utf8(), False), pa.field("dept_id", pa.int64(), False)]
        ),
    )


# (name, join type, expected rows, expected columns or None) — hash_join.rs:710-743
JOIN_CASES = [
    ("test_inner_join", JoinType.Inner, 3, 5),
    ("test_left_semi_join", JoinType.LeftSemi, 3, 3),
    ("test_left_anti_join", JoinType.LeftAnti, 1, None),
]


def join_config(jt: JoinType) -> HashJoinConfig:
    return HashJoinConfig(join_type=jt, probe_keys=[2], build_keys=[0])


# ----------------------------------------------------------- aggregate -----
# native/prism-executor/src/hash_aggregate.rs:534-552
def sales_batch() -> pa.RecordBatch:
    return pa.RecordBatch.from_arrays(
        [
            pa.array(["east", "west", "east", "west", "east"]),
            pa.array(["A", "B", "A", "A", "B"]),
            pa.array([100.0, 200.0, 150.0, 300.0, 50.0]),
            pa.array([10, 20, 15, 30, 5], pa.int64()),
        ],
        schema=pa.schema(
            [
                pa.field("region", pa.utf8(), False),
                pa.field("product", pa.utf8(), False),
                pa.field("amount", pa.float64(), False),
                pa.field("qty", pa.int64(), False),
            ]
        ),
    )


# hash_aggregate.rs:555-570: 2 rows, 2 columns, amounts total 800.0
SUM_BY_REGION = HashAggConfig(group_by=[0], aggregates=[AggExpr(2, AggFunc.Sum, "total_amount")])
# hash_aggregate.rs:573-584: 2 rows, 3 columns
COUNT_AND_AVG = HashAggConfig(
    group_by=[0],
    aggregates=[AggExpr(2, AggFunc.Count, "cnt"), AggExpr(2, AggFunc.Avg, "avg_amount")],
)


# hash_aggregate.rs:587-615: global COUNT DISTINCT over {2^53, 2^53+1, 2^53, null} = 2
def large_int64_batch() -> pa.RecordBatch:
    return pa.RecordBatch.from_arrays(
        [pa.array([9_007_199_254_740_992, 9_007_199_254_740_993, 9_007_199_254_740_992, None], pa.int64())],
        schema=pa.schema([pa.field("id", pa.int64(), True)]),
    )


GLOBAL_COUNT_DISTINCT = HashAggConfig(group_by=[], aggregates=[AggExpr(0, AggFunc.CountDistinct, "distinct_ids")])


# hash_aggregate.rs:618-660: grouped Utf8 COUNT DISTINCT: east=2, west=2
def labels_batch() -> pa.RecordBatch:
    return pa.RecordBatch.from_arrays(
        [
            pa.array(["east", "east", "east", "west", "west", "west"]),
            pa.array(["A", "A", "B", "A", None, "C"]),
        ],
        schema=pa.schema([pa.field("region", pa.utf8(), False), pa.field("label", pa.utf8(), True)]),
    )


GROUPED_COUNT_DISTINCT = HashAggConfig(group_by=[0], aggregates=[AggExpr(1, AggFunc.CountDistinct, "distinct_labels")])


# -------------------------------------------------------- filter/project ---
# native/prism-executor/src/filter_project.rs:413-431
def fp_test_batch() -> pa.RecordBatch:
    return pa.RecordBatch.from_arrays(
        [
            pa.array([1, 2, 3, 4, 5], pa.int64()),
            pa.array(["alice", "bob", "carol", "dave", "eve"]),
            pa.array([10.0, 20.0, 30.0, 40.0, 50.0]),
        ],
        schema=pa.schema([pa.field("id", pa.int64(), False), pa.field("name", pa.utf8(), False), pa.field("value", pa.float64(), False)]),
    )


# filter_project.rs:476-485: Gt(0, 3) keeps ids [4, 5]
FILTER_GT = Predicate.Gt(0, ScalarValue.Int64(3))
# filter_project.rs:488-497: Le(2, 30.0) then project [1, 2]: 3 rows, 2 cols, names alice..carol
FILTER_LE = Predicate.Le(2, ScalarValue.Float64(30.0))
# filter_project.rs:500-509: Ge(0,2) AND Le(0,4) keeps 3 rows
COMPOUND = Predicate.And(Predicate.Ge(0, ScalarValue.Int64(2)), Predicate.Le(0, ScalarValue.Int64(4)))


# filter_project.rs:434-465: CASE WHEN id = 1 THEN 'owner' ELSE label END -> owner, b, c
def if_then_batch() -> pa.RecordBatch:
    return pa.RecordBatch.from_arrays(
        [pa.array([1, 2, 3], pa.int64()), pa.array(["a", "b", "c"])],
        schema=pa.schema([pa.field("id", pa.int64(), False), pa.field("label", pa.utf8(), False)]),
    )


IF_THEN_EXPR = ScalarExpr.IfThen(
    [(Predicate.Eq(0, ScalarValue.Int64(1)), ScalarExpr.Literal(ScalarValue.Utf8("owner")))],
    ScalarExpr.ColumnRef(1),
)


# ------------------------------------------------ fused join -> aggregate --
# native/prism-substrait/src/executor.rs:903-1009
def fused_left_batches():
    schema = pa.schema(
        [pa.field("l_orderkey", pa.int64(), False), pa.field("l_extendedprice", pa.float64(), False), pa.field("l_discount", pa.float64(), False)]
    )
    return [
        pa.RecordBatch.from_arrays([pa.array([0, 1], pa.int64()), pa.array([100.0, 200.0]), pa.array([0.10, 0.20])], schema=schema),
        pa.RecordBatch.from_arrays([pa.array([2, 3], pa.int64()), pa.array([300.0, 400.0]), pa.array([0.00, 0.25])], schema=schema),
    ]


def fused_right_batch():
    return pa.RecordBatch.from_arrays(
        [pa.array([0, 1, 2, 3], pa.int64()), pa.array(["F", "F", "O", "O"])],
        schema=pa.schema([pa.field("o_orderkey", pa.int64(), False), pa.field("o_orderstatus", pa.utf8(), False)]),
    )


# Project columns [4] (o_orderstatus) + expr l_extendedprice * (1 - l_discount);
# aggregate group_by [0]: SUM(expr) , COUNT(expr)
FUSED_PROJECT_COLS = [4]
FUSED_EXPRS = [
    ScalarExpr.BinaryOp(
        ArithmeticOp.Multiply,
        ScalarExpr.ColumnRef(1),
        ScalarExpr.BinaryOp(ArithmeticOp.Subtract, ScalarExpr.Literal(ScalarValue.Float64(1.0)), ScalarExpr.ColumnRef(2)),
    )
]
FUSED_AGG = HashAggConfig(group_by=[0], aggregates=[AggExpr(1, AggFunc.Sum, "agg_0"), AggExpr(1, AggFunc.Count, "agg_1")])
FUSED_EXPECTED = {"F": (100.0 * 0.9 + 200.0 * 0.8, 2), "O": (300.0 + 400.0 * 0.75, 2)}


# executor.rs:1012-1080: AVG over a direct join input: F=15, O=35
def fused_avg_left():
    return [
        pa.RecordBatch.from_arrays(
            [pa.array([0, 1, 2, 3], pa.int64()), pa.array([10.0, 20.0, 30.0, 40.0])],
            schema=pa.schema([pa.field("l_orderkey", pa.int64(), False), pa.field("l_extendedprice", pa.float64(), False)]),
        )
    ]


# The reference's direct-join case projects the referenced columns (1, 3) in
# ascending order (fused_identity_projection, executor.rs:460-472), remapping
# group_by [3] -> [1] and the AVG column 1 -> [0].
FUSED_AVG_COLS = [1, 3]
FUSED_AVG_AGG = HashAggConfig(group_by=[1], aggregates=[AggExpr(0, AggFunc.Avg, "agg_0")])
FUSED_AVG_EXPECTED = {"F": 15.0, "O": 35.0}


# ------------------------------------------- distributed partial merge -----
# native/prism-bench/src/handler.rs:1378-1460 (merge of worker partials)
def partial_batches():
    schema = pa.schema(
        [
            pa.field("status", pa.utf8(), False),
            pa.field("agg_0", pa.float64(), True),
            pa.field("agg_1", pa.int64(), True),
            pa.field("agg_2", pa.float64(), True),
            pa.field("agg_3", pa.int64(), True),
        ]
    )
    a = pa.RecordBatch.from_arrays(
        [pa.array(["F", "O"]), pa.array([100.0, 50.0]), pa.array([2, 1], pa.int64()), pa.array([100.0, 50.0]), pa.array([2, 1], pa.int64())],
        schema=schema,
    )
    b = pa.RecordBatch.from_arrays(
        [pa.array(["F", "P"]), pa.array([30.0, 70.0]), pa.array([1, 2], pa.int64()), pa.array([30.0, 70.0]), pa.array([1, 2], pa.int64())],
        schema=schema,
    )
    return [a, b]


# build_final_merge_config(1, [Sum, Count, Sum, Count]) (executor.rs:714-743)
MERGE_CONFIG = HashAggConfig(
    group_by=[0],
    aggregates=[
        AggExpr(1, AggFunc.Sum, "agg_0"),
        AggExpr(2, AggFunc.Sum, "agg_1"),
        AggExpr(3, AggFunc.Sum, "agg_2"),
        AggExpr(4, AggFunc.Sum, "agg_3"),
    ],
)
# the original aggregates of that test (handler.rs:1379-1395): SUM, COUNT, AVG of column 1
MERGE_ORIGINAL = HashAggConfig(
    group_by=[0],
    aggregates=[AggExpr(1, AggFunc.Sum, "agg_0"), AggExpr(1, AggFunc.Count, "agg_1"), AggExpr(1, AggFunc.Avg, "agg_2")],
)
# after reconstruct: F=(130, 3, 130/3), O=(50, 1, 50), P=(70, 2, 35)
MERGE_EXPECTED = {"F": (130.0, 3, 130.0 / 3.0), "O": (50.0, 1, 50.0), "P": (70.0, 2, 35.0)}


# ---------------------------------------------------------------- sort -----
# native/prism-executor/src/sort.rs:238-253 (test_batch)
def sort_test_batch() -> pa.RecordBatch:
    schema = pa.schema([pa.field("name", pa.utf8(), nullable=False), pa.field("age", pa.int64(), nullable=False),
                        pa.field("score", pa.float64(), nullable=False)])
    return pa.RecordBatch.from_arrays(
        [pa.array(["Charlie", "Alice", "Bob", "Dave", "Eve"]), pa.array([30, 25, 25, 35, 28], pa.int64()),
         pa.array([85.5, 92.0, 88.0, 76.0, 92.0])], schema=schema)


# sort.rs:255-266 test_sort_by_name_asc: names[0] == "Alice", names[4] == "Eve"
SORT_BY_NAME_ASC = [SortKey(0, SortDirection.Asc, NullOrdering.NullsLast)]
# sort.rs:268-279 test_sort_by_score_desc_limit: 3 rows, scores[0] == 92.0
SORT_BY_SCORE_DESC = [SortKey(2, SortDirection.Desc, NullOrdering.NullsLast)]
# sort.rs:281-299 test_multi_key_sort: ages[0] == 25, scores[0] == 92.0
SORT_MULTI_KEY = [SortKey(1, SortDirection.Asc, NullOrdering.NullsLast),
                  SortKey(2, SortDirection.Desc, NullOrdering.NullsLast)]
