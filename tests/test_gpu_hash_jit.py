"""Run-time generated hashed-groups aggregation kernels against the oracle.

GROUP BY over hashed keys (integers, floats, strings, several columns) runs a
generated kernel whose per-block shared-memory table slots own their
accumulator words. These cases cover key types and nulls, group counts that
fit one block's table and counts that overflow it into the global table,
the filter/projection fused in front, both arithmetic modes, and check that
the generated kernel is the one that ran.
"""
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


def keyed(n, seed, groups, nulls):
    """k int64 (`groups` distinct), k32 int32, kf float64 (with -0.0, +0.0,
    NaN), ks utf8, v int64, x float64."""
    rng = np.random.default_rng(seed)

    def mask(p):
        return (rng.random(n) < p) if nulls else None

    pool = rng.integers(-(2**62), 2**62, groups)
    fpool = np.concatenate([rng.normal(0, 1e3, max(1, groups - 3)), [0.0, -0.0, np.nan]])
    spool = np.array([f"key-{i:06d}-{'x' * (i % 23)}" for i in range(groups)])
    x = rng.normal(0, 5, n)
    x[rng.random(n) < 0.005] = np.nan
    return pa.RecordBatch.from_arrays(
        [
            pa.array(pool[rng.integers(0, groups, n)], mask=mask(0.03)),
            pa.array(rng.integers(-40, 40, n).astype(np.int32), mask=mask(0.03)),
            pa.array(fpool[rng.integers(0, len(fpool), n)], mask=mask(0.03)),
            pa.array(spool[rng.integers(0, groups, n)], mask=mask(0.03)),
            pa.array(rng.integers(-10**9, 10**9, n), mask=mask(0.05)),
            pa.array(x, mask=mask(0.05)),
        ],
        names=["k", "k32", "kf", "ks", "v", "x"],
    )


AGGS = [(4, AggFunc.Count), (4, AggFunc.Sum), (4, AggFunc.Min), (4, AggFunc.Max), (5, AggFunc.Sum), (5, AggFunc.Avg)]
KEYS = {"int64": [0], "int32": [1], "float64": [2], "utf8": [3], "int32+utf8": [1, 3], "int64+float64": [0, 2]}


def cfg(keys, aggs=AGGS):
    return HashAggConfig(list(keys), [AggExpr(c, f, f"a{i}") for i, (c, f) in enumerate(aggs)])


def float_cols(ref):
    return tuple(i for i in range(ref.num_columns) if pa.types.is_floating(ref.schema.field(i).type))


@pytest.fixture
def prof(ctx):
    ctx.set_profiling(True)
    yield ctx
    ctx.set_profiling(False)


def ran(ctx, before):
    return ctx.kernel_stats("agg_hash_jit")[0] - before


@pytest.mark.parametrize("nulls", [False, True])
@pytest.mark.parametrize("key", sorted(KEYS))
def test_hashed_groups(prof, key, nulls):
    bs = [keyed(60_000, 31 + k, 700, nulls) for k in range(2)]
    c = cfg(KEYS[key])
    before = prof.kernel_stats("agg_hash_jit")[0]
    got = prism_gpu.hash_aggregate_batches(bs, c, ctx=prof)
    assert ran(prof, before) == len(bs)
    ref = oracle.hash_aggregate_batches(bs, c, n_threads=2)
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


@pytest.mark.parametrize("groups", [1, 3000, 60_000])
def test_group_counts_past_the_block_table(prof, groups):
    """More groups than a block's table holds: rows overflow to the global
    table (and the global table regrows), results unchanged."""
    bs = [keyed(150_000, 41, groups, True)]
    c = cfg([0])
    before = prof.kernel_stats("agg_hash_jit")[0]
    got = prism_gpu.hash_aggregate_batches(bs, c, ctx=prof)
    assert ran(prof, before) >= 1
    ref = oracle.hash_aggregate_batches(bs, c, n_threads=2)
    assert got.num_rows == ref.num_rows
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


@pytest.mark.parametrize("mode", [ARITH_F64, ARITH_EXACT])
def test_fused_filter_and_expressions(prof, mode):
    bs = [keyed(80_000, 51 + k, 900, True) for k in range(2)]
    pred = P.And(P.Gt(4, S.Int64(-600_000_000)), P.Not(P.Eq(1, S.Int32(7))))
    ex = [E.BinaryOp(Op.Multiply, E.ColumnRef(4), E.BinaryOp(Op.Subtract, E.Literal(S.Int64(100)), E.ColumnRef(1)))]
    # projected schema: [k, k32, v, x, expr_0]
    c = HashAggConfig([0, 1], [AggExpr(4, AggFunc.Sum, "s"), AggExpr(4, AggFunc.Avg, "a"), AggExpr(2, AggFunc.Count, "n"),
                               AggExpr(3, AggFunc.Min, "mn")] if mode == ARITH_F64 else
                      [AggExpr(4, AggFunc.Sum, "s"), AggExpr(2, AggFunc.Sum, "sv"), AggExpr(2, AggFunc.Count, "n")])
    before = prof.kernel_stats("agg_hash_jit")[0]
    got = prism_gpu.filter_project_aggregate(bs, pred, [0, 1, 4, 5], ex, c, arith_mode=mode, ctx=prof)
    assert ran(prof, before) == len(bs)
    ref = oracle.filter_project_aggregate(bs, pred, [0, 1, 4, 5], ex, c, arith_mode=mode, n_threads=2)
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


def test_int64_sum_limbs_exact(prof):
    """Integer sums near the int64 edges: the two 32-bit limbs carry exactly."""
    n = 200_000
    rng = np.random.default_rng(9)
    k = pa.array(rng.integers(0, 500, n))
    v = pa.array(np.where(rng.random(n) < 0.5, np.int64(2**63 - 1), np.int64(-(2**63))))
    b = pa.RecordBatch.from_arrays([k, v], names=["k", "v"])
    c = cfg([0], [(1, AggFunc.Sum), (1, AggFunc.Count), (1, AggFunc.Max)])
    got = prism_gpu.hash_aggregate(b, c, ctx=prof)
    ref = oracle.hash_aggregate(b, c, n_threads=2)
    assert_batches_equal(got, ref, float_cols=float_cols(ref))
