"""Fused filter->project->aggregate and join->aggregate against the oracle."""
import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from golden import reference_kat as K
from helpers import assert_batches_equal
from prism_gpu import ARITH_EXACT, AggExpr, AggFunc, ArithmeticOp, HashAggConfig, Predicate, ScalarExpr, ScalarValue

pytestmark = pytest.mark.gpu

S = ScalarValue


def lineitem(n, seed):
    """100M-row fact-table shape at small n: quantity, price (cents), discount
    and tax (hundredths), ship_day, flag/status dictionaries."""
    rng = np.random.default_rng(seed)
    return pa.RecordBatch.from_arrays(
        [
            pa.array(rng.integers(1, 51, n)),
            pa.array(rng.integers(90_000, 10_500_001, n)),
            pa.array(rng.integers(0, 11, n)),
            pa.array(rng.integers(0, 9, n)),
            pa.array(rng.integers(0, 2526, n).astype(np.int32)),
            pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 3, n).astype(np.int8)), pa.array(["A", "N", "R"])),
            pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 2, n).astype(np.int8)), pa.array(["F", "O"])),
        ],
        names=["quantity", "price", "discount", "tax", "ship_day", "flag", "status"],
    )


def c(i):
    return ScalarExpr.ColumnRef(i)


def L(v):
    return ScalarExpr.Literal(S.Int64(v))


DISC = ScalarExpr.BinaryOp(ArithmeticOp.Multiply, c(1), ScalarExpr.BinaryOp(ArithmeticOp.Subtract, L(100), c(2)))
CHARGE = ScalarExpr.BinaryOp(ArithmeticOp.Multiply, DISC, ScalarExpr.BinaryOp(ArithmeticOp.Add, L(100), c(3)))
FILTER = Predicate.Le(4, S.Int32(2436))
COLS = [5, 6]
AGG = HashAggConfig(
    [0, 1],
    [
        AggExpr(2, AggFunc.Sum, "sum_disc_price"),
        AggExpr(2, AggFunc.Avg, "avg_disc_price"),
        AggExpr(3, AggFunc.Sum, "sum_charge"),
        AggExpr(3, AggFunc.Avg, "avg_charge"),
        AggExpr(2, AggFunc.Count, "count_order"),
    ],
)


@pytest.mark.parametrize("mode", [prism_gpu.ARITH_F64, ARITH_EXACT])
def test_filter_project_aggregate_shape(ctx, mode):
    bs = [lineitem(120_000, s) for s in range(3)]
    got = prism_gpu.filter_project_aggregate(bs, FILTER, COLS, [DISC, CHARGE], AGG, arith_mode=mode)
    ref = oracle.filter_project_aggregate(bs, FILTER, COLS, [DISC, CHARGE], AGG, arith_mode=mode, n_threads=2)
    assert_batches_equal(got, ref, float_cols=(2, 3, 4, 5))
    if mode == ARITH_EXACT:
        assert pa.types.is_decimal(got.schema.field(2).type)
        assert got.column(2).equals(ref.column(2)) and got.column(4).equals(ref.column(4))


def test_exact_sums_match_reference_f64_within_tolerance(ctx):
    bs = [lineitem(200_000, 9)]
    exact = prism_gpu.filter_project_aggregate(bs, FILTER, COLS, [DISC, CHARGE], AGG, arith_mode=ARITH_EXACT)
    ref = oracle.filter_project_aggregate(bs, FILTER, COLS, [DISC, CHARGE], AGG)
    for i in (2, 4):
        e = np.array([float(x) * 10 ** exact.schema.field(i).type.scale for x in exact.column(i).to_pylist()])
        r = ref.column(i).to_numpy()
        assert np.all(np.abs(e - r) <= 1e-12 * np.abs(r))


def test_fused_join_aggregate_known_answers(ctx):
    out = prism_gpu.join_aggregate(K.fused_left_batches(), K.fused_right_batch(), [0], [0], K.FUSED_PROJECT_COLS, K.FUSED_EXPRS, K.FUSED_AGG)
    rows = {s: (v, n) for s, v, n in zip(*(out.column(i).to_pylist() for i in range(3)))}
    assert rows == K.FUSED_EXPECTED
    out = prism_gpu.join_aggregate(K.fused_avg_left(), K.fused_right_batch(), [0], [0], K.FUSED_AVG_COLS, [], K.FUSED_AVG_AGG)
    assert dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist())) == K.FUSED_AVG_EXPECTED


def test_join_aggregate_string_keys(ctx):
    rng = np.random.default_rng(4)
    nb = 20_000
    lens = rng.integers(8, 33, nb)
    keys = ["".join(chr(97 + x) for x in rng.integers(0, 26, l)) + f"{i}" for i, l in enumerate(lens)]
    build = pa.RecordBatch.from_arrays([pa.array(keys), pa.array(rng.integers(0, 25, nb).astype(np.int32))], names=["key", "group_id"])
    probes = []
    for s in range(3):
        r = np.random.default_rng(100 + s)
        pick = r.integers(0, nb, 50_000)
        ks = [keys[i] if r.random() < 0.95 else "zz-miss-" + keys[i] for i in pick]
        probes.append(pa.RecordBatch.from_arrays([pa.array(ks), pa.array(r.lognormal(5, 1, 50_000))], names=["key", "amount"]))
    agg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "sum_amount"), AggExpr(1, AggFunc.Count, "cnt")])
    cols = [3, 1]  # group_id (build side), amount (probe side)
    got = prism_gpu.join_aggregate(probes, build, [0], [0], cols, [], agg)
    ref = oracle.join_aggregate(probes, build, [0], [0], cols, [], agg)
    assert_batches_equal(got, ref, float_cols=(1,))
