"""Run-time generated small-groups aggregation kernels against the oracle.

GROUP BY over dictionary columns with at most 8 groups runs one generated
kernel per query shape (filter, expressions and operands compiled to
straight-line code); these cases cover every predicate and expression node
kind, nullable and null-free columns, and check that the generated kernel is
the one that ran. With run-time compilation switched off the interpreting
kernel must give the same results.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from helpers import assert_batches_equal
from prism_gpu import ARITH_EXACT, ARITH_F64, AggExpr, AggFunc, HashAggConfig
from prism_gpu import ArithmeticOp as Op
from prism_gpu import Predicate as P
from prism_gpu import ScalarExpr as E
from prism_gpu import ScalarValue as S

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def table(n, seed, nulls):
    """a int64, b int32, x float64, y float32, s utf8, flag/status dictionaries."""
    rng = np.random.default_rng(seed)

    def mask(p):
        return (rng.random(n) < p) if nulls else None

    words = np.array(["alpha", "beta", "gamma", "zz", "abacus", "", "tab"])
    x = rng.normal(0, 3, n)
    x[rng.random(n) < 0.01] = np.nan
    return pa.RecordBatch.from_arrays(
        [
            pa.array(rng.integers(-10**12, 10**12, n), mask=mask(0.05)),
            pa.array(rng.integers(-200, 200, n).astype(np.int32), mask=mask(0.05)),
            pa.array(x, mask=mask(0.05)),
            pa.array(rng.normal(0, 1, n).astype(np.float32)),
            pa.array(words[rng.integers(0, len(words), n)], mask=mask(0.05)),
            pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 3, n).astype(np.int8), mask=mask(0.03)),
                                           pa.array(["A", "N", "R"])),
            pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 2, n).astype(np.int8)), pa.array(["F", "O"])),
        ],
        names=["a", "b", "x", "y", "s", "flag", "status"],
    )


def c(i):
    return E.ColumnRef(i)


def bin_(op, l, r):
    return E.BinaryOp(op, l, r)


F64_CASES = {
    "cmp_and_not": (
        P.And(P.Gt(2, S.Float64(-1.5)), P.Not(P.Lt(1, S.Int32(-50)))),
        [bin_(Op.Subtract, bin_(Op.Multiply, c(0), E.Literal(S.Float64(2.5e-9))), c(2)),
         E.IfThen([(P.Lt(1, S.Int32(0)), c(2)), (P.Eq(4, S.Utf8("zz")), c(3))], E.Negate(c(3)))],
    ),
    "strings_or_null": (
        P.Or(P.Like(4, "%ab%"), P.Or(P.IsNull(2), P.Ge(4, S.Utf8("gamma")))),
        [bin_(Op.Divide, c(2), bin_(Op.Add, c(3), E.Literal(S.Float64(10.0)))),
         E.IfThen([(P.IsNotNull(0), bin_(Op.Multiply, c(1), c(1)))])],
    ),
    "no_filter": (None, [bin_(Op.Add, c(2), c(3)), bin_(Op.Multiply, c(1), E.Literal(S.Float64(0.5)))]),
}

EXACT_CASES = {
    "products": (
        P.Le(1, S.Int32(150)),
        [bin_(Op.Multiply, c(0), bin_(Op.Subtract, E.Literal(S.Int64(100)), c(1))),
         bin_(Op.Add, E.Negate(c(0)), bin_(Op.Multiply, c(1), c(1)))],
    ),
    "select_and_literal": (
        P.Not(P.IsNull(1)),
        [E.IfThen([(P.Gt(1, S.Int32(0)), c(0))], bin_(Op.Subtract, c(1), E.Literal(S.Int64(7)))),
         bin_(Op.Multiply, bin_(Op.Multiply, c(1), c(1)), bin_(Op.Multiply, c(1), E.Literal(S.Int64(-3))))],
    ),
}


def agg_for(mode):
    # projected schema: [flag, status, a, b, x, expr_0, expr_1]; Float64
    # queries group by flag alone (up to 4 groups) so their 6 accumulators
    # per group stay within the generated kernel's register budget
    aggs = [AggExpr(5, AggFunc.Sum, "s0"), AggExpr(5, AggFunc.Avg, "a0"), AggExpr(6, AggFunc.Sum, "s1"),
            AggExpr(2, AggFunc.Sum, "sa"), AggExpr(6, AggFunc.Count, "n1")]
    if mode == ARITH_F64:
        aggs += [AggExpr(5, AggFunc.Min, "mn"), AggExpr(6, AggFunc.Max, "mx"), AggExpr(4, AggFunc.Sum, "sx")]
        return HashAggConfig([0], aggs)
    return HashAggConfig([0, 1], aggs)


def run_both(ctx, batches, pred, exprs, mode):
    cols = [5, 6, 0, 1, 2]
    agg = agg_for(mode)
    before = ctx.kernel_stats("agg_tiny_jit")[0]
    got = prism_gpu.filter_project_aggregate(batches, pred, cols, exprs, agg, arith_mode=mode, ctx=ctx)
    ran = ctx.kernel_stats("agg_tiny_jit")[0] - before
    ref = oracle.filter_project_aggregate(batches, pred, cols, exprs, agg, arith_mode=mode, n_threads=2)
    return got, ref, ran


def float_cols(ref):
    return tuple(i for i in range(ref.num_columns) if pa.types.is_floating(ref.schema.field(i).type))


@pytest.fixture
def prof(ctx):
    ctx.set_profiling(True)
    yield ctx
    ctx.set_profiling(False)


@pytest.mark.parametrize("nulls", [False, True])
@pytest.mark.parametrize("case", sorted(F64_CASES))
def test_generated_kernel_f64(prof, case, nulls):
    pred, exprs = F64_CASES[case]
    bs = [table(70_000, 11 + k, nulls) for k in range(2)]
    got, ref, ran = run_both(prof, bs, pred, exprs, ARITH_F64)
    assert ran == len(bs)
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


@pytest.mark.parametrize("nulls", [False, True])
@pytest.mark.parametrize("case", sorted(EXACT_CASES))
def test_generated_kernel_exact(prof, case, nulls):
    pred, exprs = EXACT_CASES[case]
    bs = [table(70_000, 21 + k, nulls) for k in range(2)]
    got, ref, ran = run_both(prof, bs, pred, exprs, ARITH_EXACT)
    assert ran == len(bs), (prism_gpu.jit_stats(), prof.kernel_stats("agg_kernel"))
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


def test_literal_change_reuses_kernel(prof):
    """Queries that differ only in literal values share one compiled kernel."""
    bs = [table(30_000, 5, False)]
    for lim in (-20, 40, 170):
        pred = P.Le(1, S.Int32(lim))
        exprs = [bin_(Op.Multiply, c(0), bin_(Op.Subtract, E.Literal(S.Int64(lim)), c(1))), c(1)]
        got, ref, ran = run_both(prof, bs, pred, exprs, ARITH_EXACT)
        assert ran == 1
        assert_batches_equal(got, ref, float_cols=float_cols(ref))


INTERPRETED = r"""
import json, sys
sys.path[:0] = [{paths}]
import pyarrow as pa
import prism_gpu, oracle_py as oracle
from helpers import assert_batches_equal
from test_gpu_jit import EXACT_CASES, F64_CASES, table, agg_for, float_cols
from prism_gpu import ARITH_EXACT, ARITH_F64
ctx = prism_gpu.default_context()
ctx.set_profiling(True)
cols = [5, 6, 0, 1, 2]
for mode, cases in ((ARITH_F64, F64_CASES), (ARITH_EXACT, EXACT_CASES)):
    for name, (pred, exprs) in cases.items():
        bs = [table(40_000, 3, True)]
        got = prism_gpu.filter_project_aggregate(bs, pred, cols, exprs, agg_for(mode), arith_mode=mode, ctx=ctx)
        ref = oracle.filter_project_aggregate(bs, pred, cols, exprs, agg_for(mode), arith_mode=mode, n_threads=2)
        assert_batches_equal(got, ref, float_cols=float_cols(ref))
print(json.dumps({{"jit": ctx.kernel_stats("agg_tiny_jit")[0], "interp": ctx.kernel_stats("agg_kernel")[0]}}))
"""


def test_interpreting_kernel_agrees_without_runtime_compilation():
    paths = ", ".join(repr(os.path.join(ROOT, p)) for p in ("prism-query_b200", "tests", ""))
    env = dict(os.environ, PRISM_JIT="0")
    r = subprocess.run([sys.executable, "-c", INTERPRETED.format(paths=paths)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    stats = json.loads(r.stdout.strip().splitlines()[-1])
    assert stats["jit"] == 0 and stats["interp"] > 0


def test_exact_overflow_raises_like_the_oracle(prof):
    """A 128-bit overflow in a generated exact program raises (64-bit steps
    overflow first and hand the row to the 128-bit path, which detects it)."""
    bs = [table(20_000, 8, False)]
    a4 = bin_(Op.Multiply, bin_(Op.Multiply, c(0), c(0)), bin_(Op.Multiply, c(0), c(0)))
    agg = HashAggConfig([0], [AggExpr(2, AggFunc.Sum, "s")])
    with pytest.raises(Exception) as ref_err:
        oracle.filter_project_aggregate(bs, None, [5, 6], [a4], agg, arith_mode=ARITH_EXACT, n_threads=2)
    with pytest.raises(prism_gpu.PrismError) as got_err:
        prism_gpu.filter_project_aggregate(bs, None, [5, 6], [a4], agg, arith_mode=ARITH_EXACT, ctx=prof)
    assert "overflow" in str(ref_err.value) and "overflow" in str(got_err.value)
    # rows the filter drops never raise (no row has b > 1000)
    pred = P.Gt(1, S.Int32(1000))
    got = prism_gpu.filter_project_aggregate(bs, pred, [5, 6], [a4], agg, arith_mode=ARITH_EXACT, ctx=prof)
    ref = oracle.filter_project_aggregate(bs, pred, [5, 6], [a4], agg, arith_mode=ARITH_EXACT, n_threads=2)
    assert got.num_rows == ref.num_rows == 0
