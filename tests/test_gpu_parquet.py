"""Parquet scan decoded on the GPU (prism_parquet_scan) against the oracle
(the scan logic restated from parquet_scan.rs, pyarrow decoding each row
group): the reference's own tests, then every readable type with nulls
across codecs, page versions, dictionary / PLAIN pages (including the
dictionary fallback mid-chunk), small pages, row-group and batch shapes,
projections, directories, and a scan feeding filter/project on the device.
Decoding is bit-exact: values, validity and batch boundaries must match."""
import os

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest

import oracle_py as oracle
import prism_gpu
from golden import parquet_files as PF
from prism_gpu import Predicate, ScalarValue

pytestmark = pytest.mark.gpu


def _same(got, ref):
    assert len(got) == len(ref), (len(got), len(ref))
    for g, r in zip(got, ref):
        assert g.schema == r.schema, (g.schema, r.schema)
        assert g.num_rows == r.num_rows
        for i in range(g.num_columns):
            a, b = g.column(i), r.column(i)
            assert a.null_count == b.null_count, g.schema.field(i)
            if pa.types.is_floating(a.type):  # bitwise, NaN included
                va = np.asarray(a.fill_null(0).to_numpy(zero_copy_only=False)).view(np.uint64 if a.type == pa.float64() else np.uint32)
                vb = np.asarray(b.fill_null(0).to_numpy(zero_copy_only=False)).view(np.uint64 if b.type == pa.float64() else np.uint32)
                assert np.array_equal(va, vb), g.schema.field(i)
                assert a.is_valid().equals(b.is_valid())
            else:
                assert a.equals(b), g.schema.field(i)


@pytest.fixture(scope="module")
def ref_dir(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("pq_ref_gpu"))
    PF.reference_test_file(d)
    return d


def test_reference_row_group_skipping(ctx, ref_dir):
    """test_row_group_skipping / test_parquet_scan_from_in_memory_store
    (parquet_scan.rs:639-661, 711-740): 200 rows, >= 3 of 5 row groups skipped."""
    pred = Predicate.Lt(1, ScalarValue.Float64(150.0))
    got, st = prism_gpu.parquet_scan([ref_dir], pred, ctx=ctx, with_stats=True)
    assert sum(b.num_rows for b in got) == 200
    assert st["row_groups"] == 5 and st["row_groups_skipped"] >= 3
    _same(got, oracle.parquet_scan([ref_dir], pred))


def test_reference_string_stats_skipping(ctx, ref_dir):
    """test_string_stats_skipping (parquet_scan.rs:663-685)."""
    got = prism_gpu.parquet_scan([ref_dir], Predicate.Eq(2, ScalarValue.Utf8("gamma")), ctx=ctx)
    assert sum(b.num_rows for b in got) == 100
    assert set(got[0].column(2).to_pylist()) == {"gamma"}


def test_reference_full_scan_and_empty_uris(ctx, ref_dir):
    """test_parquet_scan_empty_uris_returns_empty (parquet_scan.rs:742-756)."""
    assert prism_gpu.parquet_scan([], ctx=ctx) == []
    got = prism_gpu.parquet_scan([ref_dir], ctx=ctx)
    _same(got, oracle.parquet_scan([ref_dir]))
    assert pa.Table.from_batches(got).equals(PF.reference_test_table())


WRITE_CASES = {
    "snappy_v1_dict": dict(compression="snappy", data_page_version="1.0", use_dictionary=True),
    "snappy_v2_dict": dict(compression="snappy", data_page_version="2.0", use_dictionary=True),
    "none_v1_plain": dict(compression="none", data_page_version="1.0", use_dictionary=False),
    "snappy_v1_plain": dict(compression="snappy", data_page_version="1.0", use_dictionary=False),
    "snappy_v2_plain": dict(compression="snappy", data_page_version="2.0", use_dictionary=False),
    "small_pages_dict_fallback": dict(compression="snappy", data_page_version="1.0", use_dictionary=True,
                                      data_page_size=2048, dictionary_pagesize_limit=4096),
    "none_v2_small_pages": dict(compression="none", data_page_version="2.0", use_dictionary=True, data_page_size=1000),
}


@pytest.mark.parametrize("case", sorted(WRITE_CASES))
def test_types_encodings_codecs(ctx, tmp_path, case):
    t = PF.typed_table(30_011, seed=len(case))
    path = str(tmp_path / "t.parquet")
    pq.write_table(t, path, row_group_size=7_000, **WRITE_CASES[case])
    for batch_size in (8192, 1000, 333):
        got = prism_gpu.parquet_scan([path], batch_size=batch_size, ctx=ctx)
        _same(got, oracle.parquet_scan([path], batch_size=batch_size))
    assert pa.Table.from_batches(got).equals(t)


def test_required_columns_and_edges(ctx, tmp_path):
    t = PF.typed_table(5000, seed=3, nulls=False)
    schema = pa.schema([pa.field(f.name, f.type, False) for f in t.schema])
    t = t.cast(schema)
    path = str(tmp_path / "r.parquet")
    pq.write_table(t, path, row_group_size=1024, compression="snappy")
    _same(prism_gpu.parquet_scan([path], ctx=ctx), oracle.parquet_scan([path]))
    # all-null and empty row groups, one-row file
    e = str(tmp_path / "e.parquet")
    pq.write_table(pa.table({"x": pa.nulls(100, pa.int64()), "s": pa.nulls(100, pa.utf8())}), e, row_group_size=30)
    _same(prism_gpu.parquet_scan([e], ctx=ctx), oracle.parquet_scan([e]))
    one = str(tmp_path / "one.parquet")
    pq.write_table(pa.table({"x": [7], "s": ["only"]}), one)
    _same(prism_gpu.parquet_scan([one], ctx=ctx), oracle.parquet_scan([one]))
    empty = str(tmp_path / "none.parquet")
    pq.write_table(pa.table({"x": pa.array([], pa.int64())}), empty)
    assert prism_gpu.parquet_scan([empty], ctx=ctx) == []


def test_projection_and_expand(ctx, tmp_path):
    t = PF.typed_table(20_000, seed=9)
    path = str(tmp_path / "p.parquet")
    pq.write_table(t, path, row_group_size=6000)
    for proj, skip in (([6, 1, 3], True), ([1, 3, 6], False), ([0], False), ([2, 99], False), ([99], True),
                       (list(range(10)), False)):
        got = prism_gpu.parquet_scan([path], projection=proj, skip_expand=skip, ctx=ctx)
        _same(got, oracle.parquet_scan([path], projection=proj, skip_expand=skip))
    # an unsorted projection expands against the wrong columns, as in the reference: an error
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.parquet_scan([path], projection=[6, 1], ctx=ctx)


def test_directory_of_files_with_predicate(ctx, tmp_path):
    for k in range(3):
        t = PF.typed_table(4000, seed=20 + k)
        d = tmp_path / ("part=%d" % k)
        d.mkdir()
        pq.write_table(t, str(d / "data.parquet"), row_group_size=1000)
    (tmp_path / "_SUCCESS").write_text("")
    pred = Predicate.And(Predicate.Ge(9, ScalarValue.Int64(1500)), Predicate.Lt(9, ScalarValue.Int64(2200)))
    got, st = prism_gpu.parquet_scan([str(tmp_path)], pred, ctx=ctx, with_stats=True)
    ref = oracle.parquet_scan([str(tmp_path)], pred)
    _same(got, ref)
    assert st["files"] == 3 and st["row_groups"] == 12 and st["row_groups_skipped"] == 6


def test_scan_feeds_filter_project(ctx, tmp_path):
    """Device batches from the scan go straight into filter_and_project."""
    t = PF.typed_table(50_000, seed=4)
    path = str(tmp_path / "f.parquet")
    pq.write_table(t, path, row_group_size=20_000)
    pred = Predicate.And(Predicate.Gt(3, ScalarValue.Float64(0.0)), Predicate.Ne(6, ScalarValue.Utf8("a")))
    dev = prism_gpu.parquet_scan([path], ctx=ctx, as_device=True)
    got = [prism_gpu.filter_and_project(b, pred, [9, 3, 6], ctx=ctx) for b in dev]
    ref = [oracle.filter_and_project(b, pred, [9, 3, 6]) for b in oracle.parquet_scan([path])]
    _same(got, ref)


def test_unsupported_and_malformed(ctx, tmp_path):
    t = PF.typed_table(1000, seed=1)
    z = str(tmp_path / "z.parquet")
    pq.write_table(t, z, compression="zstd")
    with pytest.raises(prism_gpu.PrismError) as e:
        prism_gpu.parquet_scan([z], ctx=ctx)
    assert e.value.kind == "InvalidArgument"
    nested = str(tmp_path / "n.parquet")
    pq.write_table(pa.table({"l": pa.array([[1, 2], [3]])}), nested)
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.parquet_scan([nested], ctx=ctx)
    cut = str(tmp_path / "cut.parquet")
    good = str(tmp_path / "good.parquet")
    pq.write_table(t, good)
    data = open(good, "rb").read()
    open(cut, "wb").write(data[:100] + (1 << 30).to_bytes(4, "little") + b"PAR1")  # footer longer than the file
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.parquet_scan([cut], ctx=ctx)
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.parquet_scan([str(tmp_path / "nothing-here")], ctx=ctx)
    assert os.path.exists(good)


def test_prepared_decode_repeats_the_scan(ctx, tmp_path):
    """prism_parquet_prepare keeps the compressed chunks in HBM; every decode
    returns what prism_parquet_scan returns."""
    t = PF.typed_table(40_000, seed=12)
    path = str(tmp_path / "prep.parquet")
    pq.write_table(t, path, row_group_size=9_000, compression="snappy")
    pred = Predicate.Ge(9, ScalarValue.Int64(10_000))
    prep = prism_gpu.ParquetPrepared([path], pred, projection=[3, 6, 9], batch_size=4096, ctx=ctx)
    assert prep.num_rows == 40_000 - 9_000 and prep.stats["row_groups_skipped"] == 1
    assert prep.compressed_bytes > 0
    ref = oracle.parquet_scan([path], pred, projection=[3, 6, 9], batch_size=4096)
    for _ in range(2):
        got, st = prep.decode(with_stats=True)
        _same(got, ref)
        assert st["decoded_bytes"] > 0 and st["inflated_bytes"] > 0
    prep.free()


@pytest.mark.parametrize("version", ["1.0", "2.0"])
def test_long_snappy_streams(ctx, tmp_path, version):
    """Pages and dictionaries far longer than one 64 KB Snappy block (the
    streams are cut at block boundaries and inflated in parallel): sorted
    int64 (short copies reaching back 8 bytes), random bytes (long literals),
    long runs (overlapping copies), a 1 MB dictionary page."""
    rng = np.random.default_rng(77)
    n = 400_000
    t = pa.table({
        "sorted": pa.array(np.sort(rng.integers(0, 10**9, n))),
        "noise": pa.array(rng.random(n)),
        "runs": pa.array(np.repeat(rng.integers(0, 5, n // 1000), 1000)),
        "words": pa.array(np.array([f"w{i:06d}" for i in range(60_000)])[rng.integers(0, 60_000, n)]),
    })
    path = str(tmp_path / "long.parquet")
    pq.write_table(t, path, row_group_size=n, data_page_size=4 << 20, compression="snappy", data_page_version=version,
                   write_batch_size=n)
    got, st = prism_gpu.parquet_scan([path], batch_size=1 << 20, ctx=ctx, with_stats=True)
    _same(got, oracle.parquet_scan([path], batch_size=1 << 20))
    assert st["inflated_bytes"] > 4 * 65536


def _evolved_files(tmp_path):
    """Two files of one table whose schema evolved: `id` widened from int32
    to int64, `v` from float32 to float64, `name` dropped, `extra` added."""
    rng = np.random.default_rng(77)
    d = tmp_path / "evolved"
    d.mkdir()
    n1, n2 = 30_000, 25_000
    t1 = pa.table({"id": pa.array(rng.integers(-2**31, 2**31 - 1, n1).astype(np.int32)),
                   "name": pa.array([f"n{i % 113}" for i in range(n1)]),
                   "v": pa.array(rng.standard_normal(n1).astype(np.float32), mask=rng.random(n1) < 0.1)})
    big = rng.integers(-2**40, 2**40, n2)
    big[::7] = rng.integers(-30_000, 30_000, len(big[::7]))
    t2 = pa.table({"id": pa.array(big), "v": pa.array(rng.standard_normal(n2) * 1e6),
                   "extra": pa.array(rng.integers(0, 10, n2).astype(np.int32), mask=rng.random(n2) < 0.3)})
    pq.write_table(t1, d / "a.parquet", row_group_size=8_000)
    pq.write_table(t2, d / "b.parquet", row_group_size=10_000)
    return str(d)


def test_target_schema_adapts_evolved_files(ctx, tmp_path):
    """ParquetScanConfig.target_schema (parquet_scan.rs:45-50, 306-339): every
    batch of a full scan comes out in the target's fields, order and types:
    widening casts, a narrowing cast whose overflowing values become null,
    float to integer (truncated; NaN / out of range -> null), a missing column
    all null, an extra column dropped."""
    d = _evolved_files(tmp_path)
    target = pa.schema([pa.field("v", pa.float64()), pa.field("id", pa.int64(), nullable=False),
                        pa.field("extra", pa.int64()), pa.field("missing", pa.date32()),
                        pa.field("name", pa.utf8())])
    got = prism_gpu.parquet_scan([d], batch_size=7_000, target_schema=target)
    ref = oracle.parquet_scan([d], batch_size=7_000, target_schema=target)
    _same(got, ref)
    assert all(b.schema == target for b in got)
    narrow = pa.schema([pa.field("id", pa.int16()), pa.field("v", pa.int32()), pa.field("extra", pa.bool_())])
    got = prism_gpu.parquet_scan([d], batch_size=9_000, target_schema=narrow)
    _same(got, oracle.parquet_scan([d], batch_size=9_000, target_schema=narrow))
    assert sum(b.column(0).null_count for b in got) > 0  # overflowing ids became null


def test_target_schema_errors_and_projection(ctx, tmp_path):
    """A non-nullable target field that receives nulls fails (as
    RecordBatch::try_new does), a cast outside the numeric types fails; with
    a projection the batches stay file-native and expand to the target."""
    d = _evolved_files(tmp_path)
    with pytest.raises(prism_gpu.PrismError) as e:
        prism_gpu.parquet_scan([d], target_schema=pa.schema([pa.field("extra", pa.int32(), nullable=False)]))
    assert e.value.kind == "Internal"
    with pytest.raises(oracle.OracleError):
        oracle.parquet_scan([d], target_schema=pa.schema([pa.field("extra", pa.int32(), nullable=False)]))
    with pytest.raises(prism_gpu.PrismError) as e:
        prism_gpu.parquet_scan([d], target_schema=pa.schema([pa.field("name", pa.int32())]))
    assert e.value.kind == "Internal"
    f = os.path.join(d, "b.parquet")
    target = pa.schema([pa.field("id", pa.int64()), pa.field("v", pa.float64()), pa.field("extra", pa.int32()),
                        pa.field("later", pa.utf8())])
    got = prism_gpu.parquet_scan([f], projection=[1], batch_size=6_000, target_schema=target)
    _same(got, oracle.parquet_scan([f], projection=[1], batch_size=6_000, target_schema=target))
    assert got[0].schema.names == ["id", "v", "extra", "later"]
