"""GPU filter / project parity against the CPU oracle (filter_project.rs)."""
import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from golden import reference_kat as K
from helpers import assert_batches_equal
from prism_gpu import ARITH_EXACT, ArithmeticOp, Predicate, ScalarExpr, ScalarValue

pytestmark = pytest.mark.gpu

S = ScalarValue


def mixed_batch(n=20_000, seed=3):
    rng = np.random.default_rng(seed)
    m = rng.random(n) < 0.07
    words = np.array(["east_coast", "west_coast", "central", "north_west", "south_east", "Coastal", ""])
    return pa.RecordBatch.from_arrays(
        [
            pa.array(rng.integers(-50, 50, n).astype(np.int64), mask=m),
            pa.array(rng.integers(-50, 50, n).astype(np.int32)),
            pa.array(np.where(rng.random(n) < 0.01, np.nan, rng.standard_normal(n) * 10), mask=rng.random(n) < 0.05),
            pa.array(words[rng.integers(0, 7, n)], mask=rng.random(n) < 0.04),
            pa.array(rng.integers(0, 2526, n).astype(np.int32), pa.date32()),
            pa.array(rng.integers(90_000, 10_500_001, n)),
            pa.array(rng.integers(0, 11, n)),
        ],
        names=["i64", "i32", "f64", "s", "d", "price", "disc"],
    )


PREDICATES = [
    Predicate.Gt(0, S.Int64(3)),
    Predicate.Le(1, S.Int32(0)),
    Predicate.Eq(2, S.Float64(0.0)),
    Predicate.Lt(2, S.Float64(float("nan"))),
    Predicate.Ge(3, S.Utf8("east_coast")),
    Predicate.Ne(3, S.Utf8("")),
    Predicate.Le(4, S.Date32(2436)),
    Predicate.Le(4, S.Int32(100)),
    Predicate.IsNull(0),
    Predicate.IsNotNull(3),
    Predicate.And(Predicate.Ge(0, S.Int64(-10)), Predicate.Le(0, S.Int64(10))),
    Predicate.Or(Predicate.IsNull(2), Predicate.Gt(1, S.Int32(40))),
    Predicate.Not(Predicate.Eq(0, S.Int64(5))),
    Predicate.Like(3, "%coast%"),
    Predicate.ILike(3, "%COAST%"),
    Predicate.Like(3, "_ast%"),
    Predicate.Literal(False),
]


@pytest.mark.parametrize("pred", PREDICATES, ids=lambda p: p.op)
def test_predicates_and_filter(ctx, pred):
    b = mixed_batch()
    got = prism_gpu.evaluate_predicate(b, pred)
    ref = oracle.evaluate_predicate(b, pred)
    assert got.equals(ref)
    assert_batches_equal(prism_gpu.filter_batch(b, got), oracle.filter_batch(b, ref))


def test_reference_known_answers(ctx):
    b = K.fp_test_batch()
    assert prism_gpu.filter_batch(b, prism_gpu.evaluate_predicate(b, K.FILTER_GT)).column(0).to_pylist() == [4, 5]
    out = prism_gpu.filter_and_project(b, K.FILTER_LE, [1, 2])
    assert out.num_rows == 3 and out.column(0).to_pylist()[::2] == ["alice", "carol"]
    assert prism_gpu.filter_batch(b, prism_gpu.evaluate_predicate(b, K.COMPOUND)).num_rows == 3
    assert prism_gpu.project_batch_with_exprs(K.if_then_batch(), [0], [K.IF_THEN_EXPR]).column(1).to_pylist() == ["owner", "b", "c"]


def test_compare_type_errors(ctx):
    b = mixed_batch(100)
    for bad in (Predicate.Eq(0, S.Int32(1)), Predicate.Lt(2, S.Int64(1)), Predicate.Like(0, "%")):
        with pytest.raises(prism_gpu.PrismError) as e:
            prism_gpu.evaluate_predicate(b, bad)
        assert e.value.kind == "InvalidArgument"


def test_filter_and_project_variants(ctx):
    b = mixed_batch()
    p = Predicate.Gt(1, S.Int32(10))
    assert_batches_equal(prism_gpu.filter_and_project(b, p, [3, 0]), oracle.filter_and_project(b, p, [3, 0]))
    assert_batches_equal(prism_gpu.filter_and_project(b, p, []), oracle.filter_and_project(b, p, []))
    assert_batches_equal(prism_gpu.filter_and_project(b, None, [2]), oracle.filter_and_project(b, None, [2]))
    assert_batches_equal(prism_gpu.project_batch(b, [6, 5, 5]), oracle.project_batch(b, [6, 5, 5]))


def col(i):
    return ScalarExpr.ColumnRef(i)


def lit(v):
    return ScalarExpr.Literal(v)


def binop(op, a, b):
    return ScalarExpr.BinaryOp(op, a, b)


EXPRS = [
    binop(ArithmeticOp.Add, col(0), col(1)),
    binop(ArithmeticOp.Multiply, col(2), lit(S.Float64(2.5))),
    binop(ArithmeticOp.Divide, col(0), col(1)),
    binop(ArithmeticOp.Subtract, lit(S.Int64(100)), col(6)),
    ScalarExpr.Negate(col(2)),
    col(3),
    lit(S.Int64(7)),
    lit(S.Utf8("x")),
    ScalarExpr.IfThen([(Predicate.Gt(0, S.Int64(0)), col(2))], lit(S.Float64(-1.0))),
    ScalarExpr.IfThen([(Predicate.Gt(0, S.Int64(0)), lit(S.Int64(1))), (Predicate.Lt(0, S.Int64(-20)), col(2))], col(1)),
    ScalarExpr.IfThen([(Predicate.Like(3, "%coast"), col(3))], lit(S.Utf8("inland"))),
    ScalarExpr.IfThen([(Predicate.IsNull(3), lit(S.Utf8("?")))]),
    binop(ArithmeticOp.Multiply, col(5), binop(ArithmeticOp.Subtract, lit(S.Int64(100)), col(6))),
]


@pytest.mark.parametrize("k", range(len(EXPRS)))
def test_project_expressions_f64(ctx, k):
    b = mixed_batch()
    got = prism_gpu.project_batch_with_exprs(b, [0], [EXPRS[k]])
    ref = oracle.project_batch_with_exprs(b, [0], [EXPRS[k]])
    assert_batches_equal(got, ref)


def test_exact_decimal_projection(ctx):
    b = mixed_batch()
    disc = binop(ArithmeticOp.Multiply, col(5), binop(ArithmeticOp.Subtract, lit(S.Int64(100)), col(6)))
    charge = binop(ArithmeticOp.Multiply, disc, binop(ArithmeticOp.Add, lit(S.Int64(100)), col(6)))
    got = prism_gpu.project_batch_with_exprs(b, [], [disc, charge, binop(ArithmeticOp.Divide, col(5), lit(S.Int64(3)))], arith_mode=ARITH_EXACT)
    ref = oracle.project_batch_with_exprs(b, [], [disc, charge, binop(ArithmeticOp.Divide, col(5), lit(S.Int64(3)))], arith_mode=ARITH_EXACT)
    assert_batches_equal(got, ref)
    assert pa.types.is_decimal(got.schema.field(0).type)


def test_exact_overflow_is_an_error(ctx):
    big = pa.RecordBatch.from_arrays([pa.array([2**62, 3], pa.int64())], names=["x"])
    e = col(0)
    for _ in range(3):
        e = binop(ArithmeticOp.Multiply, e, col(0))
    with pytest.raises(prism_gpu.PrismError) as err:
        prism_gpu.project_batch_with_exprs(big, [], [e], arith_mode=ARITH_EXACT)
    assert err.value.kind == "Execution"
