"""Fused join -> aggregate (one generated kernel per probe batch: key lookup,
projection and aggregation of the joined rows, nothing materialized) against
the oracle, and against the materializing path.

Cases cover Utf8, multi-column and Int64 keys (dense-mode and hashed build
tables, duplicate build keys), group keys from either side, nulls on both
sides, expressions over joined columns, no GROUP BY, several probe batches,
a build key named like a probe column, no matches, and the group count past
which the materializing path takes over.
"""
import json
import os
import pickle
import subprocess
import sys

import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from helpers import assert_batches_equal
from prism_gpu import AggExpr, AggFunc, ArithmeticOp, HashAggConfig
from prism_gpu import ScalarExpr as E

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_side(nb, seed, key_kind, dups, nulls, groups=25):
    """key, group_id int32, weight float64, tag utf8."""
    rng = np.random.default_rng(seed)
    ids = np.arange(nb)
    if dups:
        ids = rng.integers(0, nb // 3, nb)
    mask = (lambda p: rng.random(nb) < p) if nulls else (lambda p: None)
    if key_kind == "utf8":
        keys = pa.array([f"k{i:07d}{'q' * (i % 13)}" for i in ids], mask=mask(0.02))
    elif key_kind == "int64_dense":
        keys = pa.array(ids.astype(np.int64) + 1_000, mask=mask(0.02))
    else:  # int64 over a wide range: hashed table
        keys = pa.array(ids.astype(np.int64) * 7_919_000_003 - 2**40, mask=mask(0.02))
    return pa.RecordBatch.from_arrays(
        [keys, pa.array(rng.integers(0, groups, nb).astype(np.int32), mask=mask(0.03)),
         pa.array(rng.lognormal(0, 1, nb), mask=mask(0.03)),
         pa.array(np.array(["x", "y", "zz", ""])[rng.integers(0, 4, nb)], mask=mask(0.03))],
        names=["key", "group_id", "weight", "tag"])


def probe_side(n, nb, seed, build, miss=0.1, nulls=False):
    """key drawn from the build keys (some missing), amount float64, qty int64."""
    rng = np.random.default_rng(seed)
    src = rng.integers(0, nb, n)
    keys = build.column(0).take(pa.array(src))
    if pa.types.is_string(keys.type):
        vals = np.array(keys.to_pylist(), dtype=object)
        vals[rng.random(n) < miss] = "MISS"
        keys = pa.array(vals.tolist(), type=pa.string())
    else:
        vals = keys.to_numpy(zero_copy_only=False).astype(np.float64)
        raw = np.where(np.isnan(vals), 0, vals).astype(np.int64)
        raw[rng.random(n) < miss] = -7
        keys = pa.array(raw, mask=(rng.random(n) < 0.02) if nulls else None)
    mask = (lambda p: rng.random(n) < p) if nulls else (lambda p: None)
    return pa.RecordBatch.from_arrays(
        [keys, pa.array(rng.lognormal(3, 1, n), mask=mask(0.03)), pa.array(rng.integers(-500, 500, n), mask=mask(0.03))],
        names=["key", "amount", "qty"])


# joined schema: probe [key, amount, qty] + build [key_right, group_id, weight, tag]
#                       0    1       2             3          4         5       6
AGG_BUILD_KEY = (
    [4, 1, 2, 5],  # projected: group_id, amount, qty, weight
    [],
    HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s_amount"), AggExpr(1, AggFunc.Count, "n"),
                        AggExpr(2, AggFunc.Sum, "s_qty"), AggExpr(3, AggFunc.Max, "mx_w"),
                        AggExpr(1, AggFunc.Avg, "avg_amount")]),
)
AGG_TWO_SIDES = (
    [6, 4, 1],  # tag (build), group_id (build), amount (probe); expr: amount * weight
    [E.BinaryOp(ArithmeticOp.Multiply, E.ColumnRef(1), E.ColumnRef(5))],
    HashAggConfig([0, 1], [AggExpr(3, AggFunc.Sum, "s_aw"), AggExpr(2, AggFunc.Min, "mn_amount")]),
)
AGG_PROBE_KEY = (
    [2, 1, 4],  # qty (probe) as the group key
    [],
    HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(2, AggFunc.Count, "n")]),
)
AGG_GLOBAL = (
    [1, 5],
    [],
    HashAggConfig([], [AggExpr(0, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Avg, "a"), AggExpr(0, AggFunc.Count, "n")]),
)
AGGS = {"build_key": AGG_BUILD_KEY, "two_sides": AGG_TWO_SIDES, "probe_key": AGG_PROBE_KEY, "global": AGG_GLOBAL}


def float_cols(ref):
    return tuple(i for i in range(ref.num_columns) if pa.types.is_floating(ref.schema.field(i).type))


@pytest.fixture
def prof(ctx):
    ctx.set_profiling(True)
    yield ctx
    ctx.set_profiling(False)


def run(ctx, probes, build, spec):
    cols, exprs, agg = spec
    before = ctx.kernel_stats("join_agg_jit")[0]
    got = prism_gpu.join_aggregate(probes, build, [0], [0], cols, exprs, agg, ctx=ctx)
    ran = ctx.kernel_stats("join_agg_jit")[0] - before
    ref = oracle.join_aggregate(probes, build, [0], [0], cols, exprs, agg, n_threads=2)
    return got, ref, ran


@pytest.mark.parametrize("key_kind", ["utf8", "int64_dense", "int64_hash"])
@pytest.mark.parametrize("dups", [False, True])
@pytest.mark.parametrize("agg", sorted(AGGS))
def test_fused_join_aggregate(prof, key_kind, dups, agg):
    if key_kind == "int64_dense" and dups:
        pytest.skip("a repeated key leaves dense mode (covered by int64_hash)")
    build = build_side(20_000, 3, key_kind, dups, nulls=True)
    probes = [probe_side(30_000, 20_000, 10 + k, build, nulls=True) for k in range(3)]
    got, ref, ran = run(prof, probes, build, AGGS[agg])
    assert ran == len(probes)
    assert got.num_rows == ref.num_rows
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


def test_multi_column_keys(prof):
    build = build_side(5_000, 4, "utf8", True, nulls=False)
    build = pa.RecordBatch.from_arrays(list(build.columns) + [pa.array(np.arange(5_000) % 3)],
                                       names=build.schema.names + ["k2"])
    probe = probe_side(40_000, 5_000, 5, build)
    probe = pa.RecordBatch.from_arrays(list(probe.columns) + [pa.array(np.random.default_rng(1).integers(0, 3, 40_000))],
                                       names=probe.schema.names + ["k2"])
    # joined: probe [key, amount, qty, k2] + build [key_right, group_id, weight, tag, k2_right]
    agg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Count, "n")])
    before = prof.kernel_stats("join_agg_jit")[0]
    got = prism_gpu.join_aggregate([probe], build, [0, 3], [0, 4], [5, 1], [], agg, ctx=prof)
    assert prof.kernel_stats("join_agg_jit")[0] - before == 1
    ref = oracle.join_aggregate([probe], build, [0, 3], [0, 4], [5, 1], [], agg, n_threads=2)
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


def test_build_key_named_like_a_probe_column(prof):
    """Grouping by the build-side key: its joined name is `key_right`."""
    build = build_side(2_000, 12, "utf8", False, nulls=True)
    probes = [probe_side(20_000, 2_000, 13, build, nulls=True)]
    spec = ([3, 1], [], HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Count, "n")]))
    got, ref, ran = run(prof, probes, build, spec)
    assert ran == 1 and got.schema.names[0] == "key_right"
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


def test_many_groups_take_the_materializing_path(prof):
    """More than 4,096 groups: the fused kernel's ordering does not take
    them, the materializing path does; results unchanged."""
    build = build_side(20_000, 6, "int64_dense", False, nulls=False, groups=9_000)
    probes = [probe_side(60_000, 20_000, 7, build)]
    got, ref, _ = run(prof, probes, build, AGG_BUILD_KEY)
    assert got.num_rows == ref.num_rows > 4096
    assert_batches_equal(got, ref, float_cols=float_cols(ref))


def test_no_matches(prof):
    """No probe key matches: the empty aggregate result (group and aggregate
    fields, no rows)."""
    build = build_side(1_000, 8, "utf8", False, nulls=False)
    probe = probe_side(5_000, 1_000, 9, build, miss=1.0)
    for spec in (AGG_BUILD_KEY, AGG_GLOBAL):
        got, ref, _ = run(prof, [probe], build, spec)
        assert got.num_rows == ref.num_rows == 0
        assert got.schema.names == ref.schema.names


MATERIALIZED = r"""
import pickle, sys
sys.path[:0] = [{paths}]
import prism_gpu
from test_gpu_join_agg import AGGS, build_side, probe_side
ctx = prism_gpu.default_context()
ctx.set_profiling(True)
build = build_side(20_000, 3, "utf8", True, nulls=True)
probes = [probe_side(30_000, 20_000, 10 + k, build, nulls=True) for k in range(2)]
out = {{name: prism_gpu.join_aggregate(probes, build, [0], [0], c, e, a, ctx=ctx) for name, (c, e, a) in AGGS.items()}}
with open({dump!r}, "wb") as f:
    pickle.dump(out, f)
print(ctx.kernel_stats("join_agg_jit")[0])
"""


def test_fused_equals_materialized(prof, tmp_path):
    """The same joins with the fused kernel switched off (joined rows
    materialized, then aggregated) give identical results."""
    paths = ", ".join(repr(os.path.join(ROOT, p)) for p in ("prism-query_b200", "tests", ""))
    dump = str(tmp_path / "materialized.pkl")
    env = dict(os.environ, PRISM_JOIN_AGG_FUSED="0")
    r = subprocess.run([sys.executable, "-c", MATERIALIZED.format(paths=paths, dump=dump)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    assert int(r.stdout.strip().splitlines()[-1]) == 0
    with open(dump, "rb") as f:
        materialized = pickle.load(f)
    build = build_side(20_000, 3, "utf8", True, nulls=True)
    probes = [probe_side(30_000, 20_000, 10 + k, build, nulls=True) for k in range(2)]
    for name, (cols, exprs, agg) in AGGS.items():
        got = prism_gpu.join_aggregate(probes, build, [0], [0], cols, exprs, agg, ctx=prof)
        assert_batches_equal(got, materialized[name], float_cols=float_cols(got))


@pytest.mark.parametrize("long_keys", [False, True])
@pytest.mark.parametrize("dups", [False, True])
def test_utf8_slot_entries(prof, monkeypatch, long_keys, dups):
    """The opt-in 64-byte slot entries (PRISM_JOIN_KEY_ENTRIES=1): keys of
    up to 32 bytes compared inside the entry, longer ones (up to 48 here)
    against the column, slots of several build rows through the row list,
    null keys on both sides, and the group_id column (no nulls) read from the
    entries."""
    monkeypatch.setenv("PRISM_JOIN_KEY_ENTRIES", "1")
    rng = np.random.default_rng(77)
    nb = 20_000
    ids = rng.integers(0, nb // 3, nb) if dups else np.arange(nb)
    pad = 40 if long_keys else 13
    keys = pa.array([f"k{i:07d}{'q' * (i % pad)}" for i in ids], mask=rng.random(nb) < 0.02)
    build = pa.RecordBatch.from_arrays(
        [keys, pa.array(rng.integers(0, 25, nb).astype(np.int32)), pa.array(rng.lognormal(0, 1, nb)),
         pa.array(np.array(["x", "y", "zz", ""])[rng.integers(0, 4, nb)])],
        names=["key", "group_id", "weight", "tag"])
    probes = [probe_side(30_000, nb, 40 + k, build) for k in range(2)]
    for spec in (AGG_BUILD_KEY, AGG_TWO_SIDES):
        got, ref, ran = run(prof, probes, build, spec)
        assert ran == len(probes)
        assert_batches_equal(got, ref, float_cols=float_cols(ref))


@pytest.mark.parametrize("dups", [False, True])
def test_utf8_unsplit_lookup(prof, monkeypatch, dups):
    """PRISM_JOIN_SPLIT=0 (the default): the fused kernel looks Utf8 keys up
    itself, no match_rows_kernel launch."""
    monkeypatch.setenv("PRISM_JOIN_SPLIT", "0")
    build = build_side(20_000, 5, "utf8", dups, nulls=True)
    probes = [probe_side(30_000, 20_000, 60 + k, build, nulls=True) for k in range(2)]
    for spec in (AGG_BUILD_KEY, AGG_TWO_SIDES, AGG_GLOBAL):
        before = prof.kernel_stats("match_rows_kernel")[0]
        got, ref, ran = run(prof, probes, build, spec)
        assert ran == len(probes)
        assert prof.kernel_stats("match_rows_kernel")[0] == before
        assert_batches_equal(got, ref, float_cols=float_cols(ref))


@pytest.mark.parametrize("entries", ["0", "1"])
def test_utf8_split_lookup_runs(prof, monkeypatch, entries):
    """PRISM_JOIN_SPLIT=1: one match_rows_kernel launch per probe batch
    (over the row records, or over the slot entries), group_id handed over
    per row (no nulls, so inlined); keys of 10-39 bytes, so some are longer
    than an entry holds."""
    monkeypatch.setenv("PRISM_JOIN_SPLIT", "1")
    monkeypatch.setenv("PRISM_JOIN_KEY_ENTRIES", entries)
    rng = np.random.default_rng(91)
    nb = 10_000
    build = pa.RecordBatch.from_arrays(
        [pa.array([f"key-{i:06d}{'z' * (i % 30)}" for i in range(nb)]),
         pa.array(rng.integers(0, 25, nb).astype(np.int32)), pa.array(rng.lognormal(0, 1, nb)),
         pa.array(np.array(["x", "y"])[rng.integers(0, 2, nb)])], names=["key", "group_id", "weight", "tag"])
    probes = [probe_side(25_000, nb, 70 + k, build) for k in range(3)]
    before = prof.kernel_stats("match_rows_kernel")[0]
    got, ref, ran = run(prof, probes, build, AGG_BUILD_KEY)
    assert prof.kernel_stats("match_rows_kernel")[0] - before == len(probes)
    assert_batches_equal(got, ref, float_cols=float_cols(ref))
