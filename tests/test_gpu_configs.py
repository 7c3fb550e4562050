"""Parity on the workload shapes themselves, at reduced sizes the oracle
finishes in seconds, with the configs' own distributions (not uniform keys):

- inner join, int64 keys: 1M unique build keys (a permutation) + int64
  payload x 10M probe keys Zipf(1.1) over 1.25M ranks through a seeded
  permutation (about 20% miss, the hottest key carrying ~12% of the probes),
  on the dense table and on the hash table; the whole output against the
  oracle's (hash_join.rs:143-200 order), and the (probe_row, payload) pairs
  of join_project as a multiset;
- join -> aggregate, Utf8 keys: 1.5M unique 8-32 byte build keys + int32
  group id over 25 values x 15M probe rows (Zipf(0.8) over the build keys,
  5% non-members), SUM(amount) within 1e-12 and COUNT bit-exact;
- filter -> project -> aggregate: 10M fact rows in EXACT mode, the int128
  sums bit-exact against the oracle's __int128 arithmetic.
"""
import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from helpers import assert_batches_equal
from prism_gpu import (ARITH_EXACT, AggExpr, AggFunc, ArithmeticOp, HashAggConfig, HashJoinConfig, JoinType, Predicate,
                       ScalarExpr, ScalarValue)

pytestmark = pytest.mark.gpu


def zipf_ranks(rng, s, n_ranks, n):
    """Ranks 0..n_ranks-1 drawn Zipf(s) by inverse CDF on the exact
    normalised weights (the generator the workloads use)."""
    w = np.arange(1, n_ranks + 1, dtype=np.float64) ** -s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), n_ranks - 1)


# ------------------------------------------------------------- int64 join --
N_BUILD, N_PROBE, N_RANKS = 1_000_000, 10_000_000, 1_250_000


@pytest.fixture(scope="module")
def c2_inputs():
    rng = np.random.default_rng(2024)
    bkeys = rng.permutation(N_BUILD).astype(np.int64)
    bpay = rng.integers(-(2**63), 2**63 - 1, N_BUILD, dtype=np.int64)
    sigma = rng.permutation(N_RANKS).astype(np.int64)
    pkeys = sigma[zipf_ranks(rng, 1.1, N_RANKS, N_PROBE)]
    ppay = rng.integers(0, 2**31 - 1, N_PROBE).astype(np.int32)
    build = pa.RecordBatch.from_arrays([pa.array(bkeys), pa.array(bpay)], names=["key", "payload"])
    probe = pa.RecordBatch.from_arrays([pa.array(pkeys), pa.array(ppay)], names=["key", "x"])
    ref = oracle.hash_join(probe, build, HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0]), n_threads=8)
    return build, probe, ref


@pytest.mark.parametrize("table", ["dense", "dense-pairs", "hash", "hash-partitioned"])
def test_c2_zipf_join_matches_oracle(ctx, c2_inputs, monkeypatch, table):
    build, probe, ref = c2_inputs
    if table == "dense-pairs":  # {row, payload} pairs in key order, one 16-byte read per probe row
        monkeypatch.setenv("PRISM_JOIN_DENSE_PAIRS", "1")
    if not table.startswith("dense"):
        monkeypatch.setenv("PRISM_JOIN_DENSE", "0")
        # the radix-partitioned build and probe forced on / off
        monkeypatch.setenv("PRISM_JOIN_PARTITION", "1" if table == "hash-partitioned" else "0")
    miss = 1 - ref.num_rows / N_PROBE
    assert 0.05 < miss < 0.4, miss  # the mass-weighted miss rate of the permuted ranks
    cfg = HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0])
    got = prism_gpu.hash_join(probe, build, cfg)
    assert_batches_equal(got, ref)

    # the workload's output, (probe_row_idx, build_payload), through the
    # resident table, in probe order and as a multiset (one-pass probe)
    t = prism_gpu.HashTable.build(build, [0], ctx)
    assert t.layout == table.split("-")[0]
    exp_rows = np.flatnonzero(np.isin(probe.column(0).to_numpy(), build.column(0).to_numpy()))
    for any_order in (False, True):
        out = t.join_project(probe, [0], [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 3], any_order=any_order)
        assert out.num_rows == ref.num_rows
        prow = out.column(0).to_numpy().astype(np.int64)
        pay = out.column(1).to_numpy()
        if any_order:
            # unique build keys: one match per probe row at most, so sorting
            # by the probe row puts the pairs in the oracle's order
            order = np.argsort(prow, kind="stable")
            prow, pay = prow[order], pay[order]
        assert np.array_equal(prow, exp_rows)
        assert np.array_equal(pay, ref.column(3).to_numpy())
    t.free()


# ------------------------------------------------------ utf8 join -> agg --
C4_BUILD, C4_PROBE, C4_BATCH = 1_500_000, 15_000_000, 1_000_000


@pytest.fixture(scope="module")
def c4_inputs():
    rng = np.random.default_rng(4004)
    lens = rng.integers(8, 33, C4_BUILD)
    boffs = np.zeros(C4_BUILD + 1, np.int64)
    np.cumsum(lens, out=boffs[1:])
    bdata = rng.integers(97, 123, int(boffs[-1]), dtype=np.uint8)
    idx = np.arange(C4_BUILD)
    for k in range(5):  # the first 5 letters spell the row index in base 26: unique keys
        bdata[boffs[:-1] + k] = (97 + (idx // 26**k) % 26).astype(np.uint8)
    build = pa.RecordBatch.from_arrays(
        [pa.Array.from_buffers(pa.utf8(), C4_BUILD, [None, pa.py_buffer(boffs.astype(np.int32)), pa.py_buffer(bdata)]),
         pa.array(rng.integers(0, 25, C4_BUILD).astype(np.int32))], names=["key", "group_id"])
    perm = rng.permutation(C4_BUILD)
    probes = []
    for _ in range(C4_PROBE // C4_BATCH):
        n = C4_BATCH
        src = perm[zipf_ranks(rng, 0.8, C4_BUILD, n)]
        plen = lens[src]
        poffs = np.zeros(n + 1, np.int64)
        np.cumsum(plen, out=poffs[1:])
        gather = np.repeat(boffs[src] - poffs[:-1], plen) + np.arange(int(poffs[-1]))
        pdata = bdata[gather]
        miss = rng.random(n) < 0.05
        pdata[poffs[:-1][miss]] = ord("Z")  # upper case never occurs in build keys
        amount = rng.lognormal(5.0, 1.0, n)
        key = pa.Array.from_buffers(pa.utf8(), n, [None, pa.py_buffer(poffs.astype(np.int32)), pa.py_buffer(pdata)])
        probes.append(pa.RecordBatch.from_arrays([key, pa.array(amount)], names=["key", "amount"]))
    agg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "sum_amount"), AggExpr(1, AggFunc.Count, "cnt")])
    ref = oracle.join_aggregate(probes, build, [0], [0], [3, 1], [], agg, n_threads=8)
    return build, probes, agg, ref


@pytest.mark.parametrize("build_path", ["default", "partitioned", "entries", "split"])
def test_c4_utf8_join_aggregate_matches_oracle(ctx, c4_inputs, monkeypatch, build_path):
    build, probes, agg, ref = c4_inputs
    if build_path == "partitioned":  # the radix-partitioned build of the Utf8 table
        monkeypatch.setenv("PRISM_JOIN_PARTITION", "1")
    if build_path == "entries":  # 64-byte slot entries carrying group_id
        monkeypatch.setenv("PRISM_JOIN_KEY_ENTRIES", "1")
    if build_path == "split":  # match_rows_kernel's per-row match words, then the aggregation
        monkeypatch.setenv("PRISM_JOIN_SPLIT", "1")
    assert ref.num_rows == 25
    got = prism_gpu.join_aggregate(probes, build, [0], [0], [3, 1], [], agg)
    # group keys and COUNT bit-exact (first-seen order), SUM within 1e-12
    assert_batches_equal(got, ref, float_cols=(1,))
    hits = sum(ref.column(2).to_pylist())
    assert 0.93 * C4_PROBE < hits < 0.97 * C4_PROBE


# ------------------------------------------- filter -> project -> agg -----
def test_c3_exact_sums_match_oracle(ctx):
    n = 10_000_000
    rng = np.random.default_rng(303)
    batches = []
    for lo in range(0, n, 2_000_000):
        m = 2_000_000
        batches.append(pa.RecordBatch.from_arrays(
            [pa.array(rng.integers(1, 51, m)), pa.array(rng.integers(90_000, 10_500_001, m)),
             pa.array(rng.integers(0, 11, m)), pa.array(rng.integers(0, 9, m)),
             pa.array(rng.integers(0, 2526, m).astype(np.int32)),
             pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 3, m).astype(np.int8)), pa.array(["A", "N", "R"])),
             pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 2, m).astype(np.int8)), pa.array(["F", "O"]))],
            names=["quantity", "price", "discount", "tax", "ship_day", "flag", "status"]))
    c = ScalarExpr.ColumnRef
    L = lambda v: ScalarExpr.Literal(ScalarValue.Int64(v))  # noqa: E731
    disc = ScalarExpr.BinaryOp(ArithmeticOp.Multiply, c(1), ScalarExpr.BinaryOp(ArithmeticOp.Subtract, L(100), c(2)))
    charge = ScalarExpr.BinaryOp(ArithmeticOp.Multiply, disc, ScalarExpr.BinaryOp(ArithmeticOp.Add, L(100), c(3)))
    agg = HashAggConfig([0, 1], [
        AggExpr(2, AggFunc.Sum, "sum_disc_price"), AggExpr(2, AggFunc.Avg, "avg_disc_price"),
        AggExpr(3, AggFunc.Sum, "sum_charge"), AggExpr(3, AggFunc.Avg, "avg_charge"), AggExpr(2, AggFunc.Count, "count_order")])
    pred = Predicate.Le(4, ScalarValue.Int32(2436))
    got = prism_gpu.filter_project_aggregate(batches, pred, [5, 6], [disc, charge], agg, arith_mode=ARITH_EXACT)
    ref = oracle.filter_project_aggregate(batches, pred, [5, 6], [disc, charge], agg, arith_mode=ARITH_EXACT, n_threads=8)
    assert got.num_rows == 6
    assert_batches_equal(got, ref, float_cols=(3, 5))
    for i in (2, 4, 6):  # the exact int128 sums and the count, bit for bit
        assert got.column(i).equals(ref.column(i))
