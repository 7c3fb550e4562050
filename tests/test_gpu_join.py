"""GPU hash join parity against the CPU oracle (hash_join.rs semantics)."""
import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from golden import reference_kat as K
from helpers import assert_batches_equal
from prism_gpu import HashJoinConfig, HashTable, JoinType

pytestmark = pytest.mark.gpu

ALL_TYPES = [JoinType.Inner, JoinType.Left, JoinType.Right, JoinType.Full, JoinType.LeftSemi, JoinType.LeftAnti]


@pytest.mark.parametrize("name,jt,rows,cols", K.JOIN_CASES)
def test_reference_known_answers(ctx, name, jt, rows, cols):
    out = prism_gpu.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(jt))
    assert out.num_rows == rows
    if cols is not None:
        assert out.num_columns == cols
    assert_batches_equal(out, oracle.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(jt)))


@pytest.mark.parametrize("jt", ALL_TYPES)
def test_all_join_types_small(ctx, jt):
    if jt == JoinType.Full:
        # the unmatched probe row (dept 99) puts a null into the non-nullable
        # build field dept_name: arrow-rs RecordBatch::try_new rejects that
        # batch in the reference, and both engines report the Arrow error
        with pytest.raises(oracle.OracleError) as e1:
            oracle.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(jt))
        with pytest.raises(prism_gpu.PrismError) as e2:
            prism_gpu.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(jt))
        assert e1.value.kind == e2.value.kind == "Arrow"
        return
    out = prism_gpu.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(jt))
    ref = oracle.hash_join(K.join_probe_side(), K.join_build_side(), K.join_config(jt))
    assert_batches_equal(out, ref)


def _int_join_batches(seed, n_build, n_probe, key_range, dup=False, nulls=False):
    rng = np.random.default_rng(seed)
    if dup:
        bkeys = rng.integers(0, max(1, n_build // 4), n_build).astype(np.int64)
    else:
        bkeys = rng.permutation(n_build).astype(np.int64)
    pkeys = rng.integers(-5, key_range, n_probe).astype(np.int64)
    bmask = (rng.random(n_build) < 0.05) if nulls else None
    pmask = (rng.random(n_probe) < 0.05) if nulls else None
    build = pa.RecordBatch.from_arrays(
        [pa.array(bkeys, mask=bmask), pa.array(rng.integers(-(2**62), 2**62, n_build)), pa.array([f"s{i % 97}" for i in range(n_build)])],
        names=["k", "payload", "label"],
    )
    probe = pa.RecordBatch.from_arrays(
        [pa.array(pkeys, mask=pmask), pa.array(rng.integers(0, 1000, n_probe).astype(np.int32))],
        names=["k", "x"],
    )
    return probe, build


@pytest.mark.parametrize("dup", [False, True])
@pytest.mark.parametrize("nulls", [False, True])
@pytest.mark.parametrize("jt", ALL_TYPES)
def test_int64_join_matches_oracle(ctx, dup, nulls, jt):
    probe, build = _int_join_batches(17, 3000, 20000, 4000, dup=dup, nulls=nulls)
    cfg = HashJoinConfig(jt, build_keys=[0], probe_keys=[0])
    assert_batches_equal(prism_gpu.hash_join(probe, build, cfg), oracle.hash_join(probe, build, cfg))


@pytest.mark.parametrize("n_build,n_probe", [(1, 1), (1, 100), (31, 33), (2047, 2049), (4096, 70000)])
def test_tile_boundaries(ctx, n_build, n_probe):
    probe, build = _int_join_batches(n_build, n_build, n_probe, n_build + 3)
    cfg = HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0])
    assert_batches_equal(prism_gpu.hash_join(probe, build, cfg), oracle.hash_join(probe, build, cfg))


def test_empty_sides(ctx):
    probe, build = _int_join_batches(5, 100, 500, 120)
    cfg = HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0])
    assert_batches_equal(prism_gpu.hash_join(probe.slice(0, 0), build, cfg), oracle.hash_join(probe.slice(0, 0), build, cfg))
    assert_batches_equal(prism_gpu.hash_join(probe, build.slice(0, 0), cfg), oracle.hash_join(probe, build.slice(0, 0), cfg))
    with pytest.raises(prism_gpu.PrismError) as e:
        prism_gpu.hash_join(probe, build.slice(0, 0), HashJoinConfig(JoinType.Left, build_keys=[0], probe_keys=[0]))
    assert e.value.kind == "Join"


def test_sentinel_and_extreme_keys(ctx):
    ks = np.array([np.iinfo(np.int64).min, -1, 0, 1, np.iinfo(np.int64).max], dtype=np.int64)
    build = pa.RecordBatch.from_arrays([pa.array(ks), pa.array(np.arange(5, dtype=np.int64))], names=["k", "v"])
    probe = pa.RecordBatch.from_arrays([pa.array(np.concatenate([ks, ks[::-1], [7]]).astype(np.int64))], names=["k"])
    cfg = HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0])
    assert_batches_equal(prism_gpu.hash_join(probe, build, cfg), oracle.hash_join(probe, build, cfg))


@pytest.mark.parametrize("partition", ["0", "1"])
def test_one_pass_hash_probe_extreme_keys(ctx, monkeypatch, partition):
    """Int64 hash slots probed by the one-pass kernel (matches as a
    multiset), streamed and radix-partitioned: the (probe_row, payload)
    pairs, the empty-slot sentinel key and the extremes included, with and
    without the build rows asked for."""
    monkeypatch.setenv("PRISM_JOIN_DENSE", "0")
    monkeypatch.setenv("PRISM_JOIN_PARTITION", partition)
    rng = np.random.default_rng(77)
    ext = np.array([np.iinfo(np.int64).min, np.iinfo(np.int64).max, -1, 0], dtype=np.int64)
    keys = np.unique(rng.integers(1, 10**12, 70_000))[:60_000]  # unique, none of the extremes
    bk = np.concatenate([ext, keys]).astype(np.int64)
    rng.shuffle(bk)
    bv = rng.integers(-(2**63), 2**63 - 1, len(bk), dtype=np.int64)
    pk = np.concatenate([rng.choice(bk, 300_000), rng.integers(1, 10**12, 100_000), ext, [ext[0]] * 3]).astype(np.int64)
    rng.shuffle(pk)
    build = pa.RecordBatch.from_arrays([pa.array(bk), pa.array(bv)], names=["k", "v"])
    probe = pa.RecordBatch.from_arrays([pa.array(pk)], names=["k"])
    pos = {int(k): i for i, k in enumerate(bk)}
    exp = sorted((r, int(bv[pos[int(k)]])) for r, k in enumerate(pk) if int(k) in pos)
    t = HashTable.build(build, [0], ctx)
    assert t.layout == "hash"
    out = t.join_project(probe, [0], [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 2], any_order=True)
    got = sorted(zip(out.column(0).to_numpy().astype(np.int64).tolist(), out.column(1).to_numpy().tolist()))
    assert got == exp
    out = t.join_project(probe, [0], [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, prism_gpu.PRISM_COL_BUILD_ROW_INDEX, 2],
                         any_order=True)
    rows = out.column(1).to_numpy().astype(np.int64)
    assert np.array_equal(bv[rows], out.column(2).to_numpy())
    got = sorted(zip(out.column(0).to_numpy().astype(np.int64).tolist(), out.column(2).to_numpy().tolist()))
    assert got == exp
    t.free()


def test_hash_table_larger_than_l2(ctx, monkeypatch):
    """5M unique Int64 keys: at the automatic load the slots (2^23, load
    0.6, 134 MB) stay larger than L2 and are probed streamed; 20M probe keys,
    80% members, as a multiset and in probe order."""
    monkeypatch.setenv("PRISM_JOIN_DENSE", "0")
    monkeypatch.setenv("PRISM_JOIN_PARTITION", "0")
    rng = np.random.default_rng(91)
    n_build, n_probe = 5_000_000, 20_000_000
    bk = rng.permutation(np.unique(rng.integers(0, 1 << 40, n_build + n_build // 8)))[:n_build].astype(np.int64)
    assert len(bk) == n_build
    bv = rng.integers(-(2**63), 2**63 - 1, n_build, dtype=np.int64)
    miss = rng.integers(1 << 40, 1 << 41, n_probe)
    pk = np.where(rng.random(n_probe) < 0.8, bk[rng.integers(0, n_build, n_probe)], miss).astype(np.int64)
    order = np.argsort(bk)
    sk = bk[order]
    at = np.minimum(np.searchsorted(sk, pk), n_build - 1)
    hit = sk[at] == pk
    exp_rows = np.flatnonzero(hit)
    exp_pay = bv[order[at[hit]]]
    build = pa.RecordBatch.from_arrays([pa.array(bk), pa.array(bv)], names=["k", "v"])
    probe = pa.RecordBatch.from_arrays([pa.array(pk)], names=["k"])
    t = HashTable.build(build, [0], ctx)
    assert t.layout == "hash"
    for any_order in (True, False):
        out = t.join_project(probe, [0], [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 2], any_order=any_order)
        rows = out.column(0).to_numpy().astype(np.int64)
        pay = out.column(1).to_numpy()
        if any_order:
            o = np.argsort(rows, kind="stable")
            rows, pay = rows[o], pay[o]
        assert np.array_equal(rows, exp_rows)
        assert np.array_equal(pay, exp_pay)
    t.free()


def test_sliced_inputs(ctx):
    probe, build = _int_join_batches(9, 1000, 5000, 1200, nulls=True)
    p2, b2 = probe.slice(3, 4000), build.slice(7, 900)
    cfg = HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0])
    assert_batches_equal(prism_gpu.hash_join(p2, b2, cfg), oracle.hash_join(p2, b2, cfg))


@pytest.mark.parametrize("jt", [JoinType.Inner, JoinType.Left, JoinType.LeftSemi, JoinType.LeftAnti])
def test_general_path_keys(ctx, jt):
    rng = np.random.default_rng(23)
    words = [f"key-{i:05d}" + "x" * (i % 29) for i in range(800)]
    bidx = rng.permutation(800)[:600]
    build = pa.RecordBatch.from_arrays(
        [pa.array([words[i] for i in bidx]), pa.array((bidx % 7).astype(np.int32)), pa.array(rng.random(600))],
        names=["s", "i", "f"],
    )
    pidx = rng.integers(0, 800, 5000)
    pmask = rng.random(5000) < 0.03
    probe = pa.RecordBatch.from_arrays(
        [pa.array([words[i] for i in pidx], mask=pmask), pa.array((pidx % 7).astype(np.int32)), pa.array(rng.integers(0, 9, 5000))],
        names=["s", "i", "z"],
    )
    for keys in ([0], [1], [0, 1]):
        cfg = HashJoinConfig(jt, build_keys=keys, probe_keys=keys)
        assert_batches_equal(prism_gpu.hash_join(probe, build, cfg), oracle.hash_join(probe, build, cfg))


def test_float_keys_nan_and_signed_zero(ctx):
    b = pa.RecordBatch.from_arrays([pa.array([0.0, -0.0, float("nan"), 1.5, 1.5]), pa.array([1, 2, 3, 4, 5])], names=["f", "v"])
    p = pa.RecordBatch.from_arrays([pa.array([0.0, -0.0, float("nan"), 1.5, 2.5])], names=["f"])
    cfg = HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0])
    assert_batches_equal(prism_gpu.hash_join(p, b, cfg), oracle.hash_join(p, b, cfg))


def test_key_type_mismatch_is_schema_error(ctx):
    b = pa.RecordBatch.from_arrays([pa.array([1, 2], pa.int64())], names=["k"])
    p = pa.RecordBatch.from_arrays([pa.array([1, 2], pa.int32())], names=["k"])
    with pytest.raises(prism_gpu.PrismError) as e:
        prism_gpu.hash_join(p, b, HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0]))
    assert e.value.kind == "SchemaMismatch"


@pytest.mark.parametrize("jt", ALL_TYPES)
def test_probe_chunked(ctx, jt):
    probe, build = _int_join_batches(31, 2000, 9000, 2600, dup=True)
    chunks = [probe.slice(0, 3000), probe.slice(3000, 0), probe.slice(3000, 6000)]
    cfg = HashJoinConfig(jt, build_keys=[0], probe_keys=[0])
    got = prism_gpu.hash_join_probe_chunked(chunks, build, cfg)
    ref = oracle.hash_join_probe_chunked(chunks, build, cfg)
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert_batches_equal(g, r)


def test_probe_matches_chunked_and_resident_table(ctx):
    probe, build = _int_join_batches(41, 5000, 30000, 6000, dup=True)
    chunks = [probe.slice(0, 10000), probe.slice(10000, 20000)]
    got = prism_gpu.probe_matches_chunked(chunks, build, [0], [0])
    ref = oracle.probe_matches_chunked(chunks, build, [0], [0])
    for g, r in zip(got, ref):
        assert g.probe_indices.equals(r.column(0)) and g.build_indices.equals(r.column(1))
    table = HashTable.build(build, [0])
    assert table.has_duplicates
    for c, r in zip(chunks, ref):
        pi, bi = table.probe(c, [0])
        assert pi.equals(r.column(0)) and bi.equals(r.column(1))


def test_join_project_emits_probe_row_and_payload(ctx):
    probe, build = _int_join_batches(51, 10000, 100000, 12500)
    table = HashTable.build(build, [0])
    out = table.join_project(probe, [0], [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 2 + 1, 1])
    ref = oracle.probe_matches_chunked([probe], build, [0], [0])[0]
    assert out.column(0).equals(ref.column(0))
    bidx = ref.column(1).to_numpy()
    assert np.array_equal(out.column(1).to_numpy(), build.column(1).to_numpy()[bidx])
    assert np.array_equal(out.column(2).to_numpy(), probe.column(1).to_numpy()[ref.column(0).to_numpy()])
    assert out.schema.names == ["probe_idx", "payload", "x"]


@pytest.mark.parametrize("mode", ["1", "0", "0p"])
def test_unique_int64_keys_dense_and_hash_tables(ctx, mode, monkeypatch):
    """Unique Int64 build keys over a compact range use the dense table
    (PRISM_JOIN_DENSE unset or 1); the hash table (0), also built by the
    radix-partitioned insert (0p), must give the same rows. A repeated key in
    a compact range falls back to the hash table."""
    monkeypatch.setenv("PRISM_JOIN_DENSE", mode[0])
    monkeypatch.setenv("PRISM_JOIN_PARTITION", "1" if mode == "0p" else "0")
    cases = [(3000, 20000, 4000, False, False), (3000, 20000, 4000, True, False), (50000, 70000, 60000, False, False),
             (3000, 9000, 4000, False, True)]
    for i, (nb, npr, kr, nulls, dup) in enumerate(cases):
        probe, build = _int_join_batches(40 + i, nb, npr, kr, dup=dup, nulls=nulls)
        for jt in (JoinType.Inner, JoinType.Left, JoinType.LeftSemi, JoinType.LeftAnti):
            cfg = HashJoinConfig(jt, build_keys=[0], probe_keys=[0])
            assert_batches_equal(prism_gpu.hash_join(probe, build, cfg), oracle.hash_join(probe, build, cfg))
    # a compact range with one key repeated
    bk = np.arange(1000, dtype=np.int64)
    bk[500] = 7
    build = pa.RecordBatch.from_arrays([pa.array(bk), pa.array(np.arange(1000, dtype=np.int64))], names=["k", "v"])
    probe = pa.RecordBatch.from_arrays([pa.array(np.arange(-3, 1003, dtype=np.int64))], names=["k"])
    cfg = HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0])
    assert_batches_equal(prism_gpu.hash_join(probe, build, cfg), oracle.hash_join(probe, build, cfg))


def _sorted_pairs(out, ncols):
    cols = [out.column(i).to_numpy() for i in range(ncols)]
    order = np.lexsort(cols[::-1])
    return [c[order] for c in cols]


@pytest.mark.parametrize("mode", ["dense", "hash", "partitioned"])
@pytest.mark.parametrize("case", ["unique", "dup", "utf8", "sliced", "tiles"])
def test_join_project_any_order_is_the_same_multiset(ctx, mode, case, monkeypatch):
    """PRISM_JOIN_ANY_ORDER: the same (probe_row, build_row, gathered
    columns) rows as the probe-order output, compared after sorting — on the
    one-pass unique-key kernel (dense table, hash table, and the hash table
    with the radix-partitioned build and probe; aligned and unaligned key
    columns, ragged tiles) and on the single-pass probe with repeated or Utf8
    keys."""
    monkeypatch.setenv("PRISM_JOIN_DENSE", "1" if mode == "dense" else "0")
    monkeypatch.setenv("PRISM_JOIN_PARTITION", "1" if mode == "partitioned" else "0")
    keys = [0]
    if case == "utf8":
        rng = np.random.default_rng(61)
        words = [f"w{i:05d}" + "y" * (i % 23) for i in range(3000)]
        build = pa.RecordBatch.from_arrays([pa.array([words[i] for i in rng.permutation(3000)[:2500]]),
                                            pa.array(rng.integers(0, 1 << 40, 2500))], names=["s", "v"])
        probe = pa.RecordBatch.from_arrays([pa.array([words[i] for i in rng.integers(0, 3000, 40000)]),
                                            pa.array(rng.integers(0, 9, 40000))], names=["s", "z"])
    elif case == "tiles":
        probe, build = _int_join_batches(62, 4000, 2048 * 7 + 1, 5000)
    else:
        probe, build = _int_join_batches(63, 20000, 150000, 26000, dup=case == "dup")
        if case == "sliced":
            probe, build = probe.slice(1, 140001), build.slice(3, 19000)
    table = HashTable.build(build, keys)
    oc = [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, prism_gpu.PRISM_COL_BUILD_ROW_INDEX, probe.num_columns + 1]
    ordered = table.join_project(probe, keys, oc)
    anyo = table.join_project(probe, keys, oc, any_order=True)
    assert anyo.num_rows == ordered.num_rows
    for a, b in zip(_sorted_pairs(anyo, 3), _sorted_pairs(ordered, 3)):
        assert np.array_equal(a, b)
    # only the probe row and one 8-byte payload: the fast emit of the one-pass kernel
    oc2 = [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, probe.num_columns + 1]
    a2 = _sorted_pairs(table.join_project(probe, keys, oc2, any_order=True), 2)
    o2 = _sorted_pairs(table.join_project(probe, keys, oc2), 2)
    for a, b in zip(a2, o2):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("graph", ["1", "0"])
def test_one_pass_probe_replayed_graph(ctx, monkeypatch, graph):
    """The one-pass probe's instantiated graph (PRISM_PROBE_GRAPH=1)
    replayed with new arguments: probes of different sizes, key alignments
    and tables on one context, back to back, each the same multiset as the
    probe-order output; and the call-by-call launch (the default) alike."""
    monkeypatch.setenv("PRISM_PROBE_GRAPH", graph)
    oc = [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 3]
    tables = []
    for dense in ("1", "0"):  # the dense and the hash kernel variants, each with its own graph
        monkeypatch.setenv("PRISM_JOIN_DENSE", dense)
        monkeypatch.setenv("PRISM_JOIN_PARTITION", "0")
        probe0, build = _int_join_batches(80 + int(dense), 20000, 10, 26000)
        tables.append((HashTable.build(build, [0], ctx), build))
    for rnd, rows in enumerate([1, 2047, 2048, 100_000, 5, 37_001]):
        for t, build in tables:
            probe, _ = _int_join_batches(90 + rnd, 20000, rows + 1, 26000)
            probe = probe.slice(rnd % 2, rows)  # aligned and unaligned key columns
            anyo = t.join_project(probe, [0], oc, any_order=True, ctx=ctx)
            ordered = t.join_project(probe, [0], oc, ctx=ctx)
            assert anyo.num_rows == ordered.num_rows
            for a, b in zip(_sorted_pairs(anyo, 2), _sorted_pairs(ordered, 2)):
                assert np.array_equal(a, b)
    for t, _ in tables:
        t.free()


@pytest.mark.parametrize("any_order", [False, True])
def test_join_project_arrow_streamed_equals_device_path(ctx, any_order):
    """prism_join_project_arrow (host batch in, host batch out) streams the
    probe in 8M-row chunks; its rows equal the device-path join_project's:
    the same rows in the same order (probe order), or the same multiset."""
    rng = np.random.default_rng(71)
    nb, npr = 300_000, 2 * (1 << 23) + 12_345  # three chunks, the last one ragged
    build = pa.RecordBatch.from_arrays([pa.array(rng.permutation(nb).astype(np.int64)),
                                        pa.array(rng.integers(-(2**62), 2**62, nb))], names=["k", "payload"])
    probe = pa.RecordBatch.from_arrays([pa.array(rng.integers(-5, int(nb * 1.25), npr).astype(np.int64)),
                                        pa.array(rng.integers(0, 1000, npr).astype(np.int32))], names=["k", "x"])
    table = HashTable.build(build, [0])
    oc = [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 3, 1, prism_gpu.PRISM_COL_BUILD_ROW_INDEX]
    got = table.join_project_arrow(probe, [0], oc, any_order=any_order)
    ref = table.join_project(probe, [0], oc)
    assert got.schema.names == ref.schema.names == ["probe_idx", "payload", "x", "build_idx"]
    assert got.num_rows == ref.num_rows
    if any_order:
        g, r = _sorted_pairs(got, 4), _sorted_pairs(ref, 4)
        for a, b in zip(g, r):
            assert np.array_equal(a, b)
    else:
        assert got.equals(ref)
    # a sliced probe batch (non-zero offset) takes the same streamed path
    sl = probe.slice(1_000_003, 9_000_000)
    assert table.join_project_arrow(sl, [0], oc).equals(table.join_project(sl, [0], oc))


def test_join_project_arrow_other_inputs_take_one_pass(ctx):
    """Repeated build keys, nullable gathered columns or Utf8 keys: one
    upload, probe and download, with the same result as the device path."""
    probe, build = _int_join_batches(72, 5000, 60000, 6000, dup=True, nulls=True)
    table = HashTable.build(build, [0])
    oc = [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 3, 4]
    assert table.join_project_arrow(probe, [0], oc).equals(table.join_project(probe, [0], oc))
    probe, build = _int_join_batches(73, 5000, 60000, 6000, nulls=True)
    table = HashTable.build(build, [0])
    assert table.join_project_arrow(probe, [0], oc).equals(table.join_project(probe, [0], oc))
    empty = probe.slice(0, 0)
    assert table.join_project_arrow(empty, [0], oc).num_rows == 0


@pytest.mark.parametrize("records", ["1", "0", "1p"])
@pytest.mark.parametrize("case", ["short", "long", "dup_nulls"])
def test_utf8_keys_packed_records_and_column_compare(ctx, records, case, monkeypatch):
    """Single Utf8 join keys compared through the packed 64-byte build key
    records (keys of at most 56 bytes) or through the build column
    (PRISM_JOIN_KEY_RECORDS=0, or a longer key anywhere): the same joins and
    join -> aggregates as the oracle, with empty strings, nulls (matched by
    keys_equal's null-flag rule) and repeated build keys."""
    monkeypatch.setenv("PRISM_JOIN_KEY_RECORDS", records[0])
    # "1p": the radix-partitioned build (row hashes partitioned, then inserted)
    monkeypatch.setenv("PRISM_JOIN_PARTITION", "1" if records == "1p" else "0")
    rng = np.random.default_rng(81)
    nb = 6000
    if case == "long":
        words = [f"k{i}" + "L" * (60 if i == 17 else i % 50) for i in range(nb)]  # one key of 62 bytes
    else:
        words = [("" if i == 0 else f"k{i:05d}" + "s" * (i % 48)) for i in range(nb)]
    bidx = rng.integers(0, nb, nb) if case == "dup_nulls" else rng.permutation(nb)
    bmask = (rng.random(nb) < 0.05) if case == "dup_nulls" else None
    build = pa.RecordBatch.from_arrays([pa.array([words[i] for i in bidx], mask=bmask),
                                        pa.array(rng.integers(0, 25, nb).astype(np.int32))], names=["k", "g"])
    pidx = rng.integers(0, nb + 500, 50_000)
    pw = [words[i] if i < nb else f"miss{i}" for i in pidx]
    pmask = (rng.random(50_000) < 0.03) if case == "dup_nulls" else None
    probe = pa.RecordBatch.from_arrays([pa.array(pw, mask=pmask), pa.array(rng.lognormal(3, 1, 50_000))],
                                       names=["k", "amount"])
    for jt in (JoinType.Inner, JoinType.Left, JoinType.LeftSemi):
        cfg = HashJoinConfig(jt, build_keys=[0], probe_keys=[0])
        assert_batches_equal(prism_gpu.hash_join(probe, build, cfg), oracle.hash_join(probe, build, cfg))
    agg = prism_gpu.HashAggConfig([0], [prism_gpu.AggExpr(1, prism_gpu.AggFunc.Sum, "s"),
                                        prism_gpu.AggExpr(1, prism_gpu.AggFunc.Count, "n")])
    got = prism_gpu.join_aggregate([probe], build, [0], [0], [3, 1], [], agg)
    assert_batches_equal(got, oracle.join_aggregate([probe], build, [0], [0], [3, 1], [], agg), float_cols=(1,))
