"""Parquet scan, host side (no GPU): the footer parser and row-group skipping
of the C library (prism_parquet_row_count reads footers only) and the
oracle's restatement, on the reference's own test file and known answers
(parquet_scan.rs:622-756)."""
import os

import pytest

import oracle_py as oracle
import prism_gpu
from golden import parquet_files as PF
from prism_gpu import Predicate, ScalarValue


@pytest.fixture(scope="module")
def ref_dir(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("pq_ref"))
    PF.reference_test_file(d)
    return d


def test_row_count_metadata(ref_dir):
    """test_row_count_metadata (parquet_scan.rs:687-709)."""
    assert prism_gpu.parquet_row_count([ref_dir]) == 500
    assert prism_gpu.parquet_row_count([ref_dir], Predicate.Lt(1, ScalarValue.Float64(150.0))) == 200


def test_statistics_skip_like_the_oracle(ref_dir):
    """row_group_might_match on every comparison / type pairing: the C
    library's row counts equal the oracle restatement's on the same file."""
    import pyarrow.parquet as pq

    f = os.path.join(ref_dir, "test.parquet")
    md = pq.ParquetFile(f).metadata
    names = pq.ParquetFile(f).schema_arrow.names
    cases = [
        Predicate.Eq(2, ScalarValue.Utf8("gamma")), Predicate.Lt(2, ScalarValue.Utf8("beta")),
        Predicate.Ge(2, ScalarValue.Utf8("epsilon")), Predicate.Gt(0, ScalarValue.Int64(399)),
        Predicate.Le(0, ScalarValue.Int64(0)), Predicate.Eq(0, ScalarValue.Int32(5)),  # Int32 vs INT64 stats: no skip
        Predicate.Eq(1, ScalarValue.Float64(250.5)), Predicate.Ne(0, ScalarValue.Int64(3)),
        Predicate.And(Predicate.Ge(0, ScalarValue.Int64(100)), Predicate.Lt(0, ScalarValue.Int64(200))),
        Predicate.Or(Predicate.Lt(0, ScalarValue.Int64(50)), Predicate.Gt(0, ScalarValue.Int64(450))),
        Predicate.Not(Predicate.Lt(0, ScalarValue.Int64(50))), Predicate.Literal(False), Predicate.IsNull(0),
        Predicate.Like(2, "%a%"), Predicate.Eq(7, ScalarValue.Int64(1)),
    ]
    for p in cases:
        want = sum(md.row_group(g).num_rows for g in range(md.num_row_groups)
                   if oracle.row_group_might_match(p, md.row_group(g), names))
        assert prism_gpu.parquet_row_count([f], p) == want, p


def test_string_stats_skip_known_answer(ref_dir):
    """test_string_stats_skipping (parquet_scan.rs:663-685): Eq(name, gamma) keeps 100 rows."""
    assert prism_gpu.parquet_row_count([ref_dir], Predicate.Eq(2, ScalarValue.Utf8("gamma"))) == 100
    assert sum(b.num_rows for b in oracle.parquet_scan([ref_dir], Predicate.Eq(2, ScalarValue.Utf8("gamma")))) == 100


def test_listing_and_errors(tmp_path, ref_dir):
    nested = tmp_path / "a" / "b"
    PF.reference_test_file(str(nested))
    (tmp_path / "a" / "notes.txt").write_text("not parquet")
    assert prism_gpu.parquet_row_count([str(tmp_path)]) == 500
    assert prism_gpu.parquet_row_count([str(tmp_path), "file://" + ref_dir]) == 1000
    assert prism_gpu.parquet_row_count([str(tmp_path / "missing")]) == 0
    bad = tmp_path / "bad.parquet"
    bad.write_bytes(b"PAR1 this is not a parquet file")
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.parquet_row_count([str(bad)])
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.parquet_row_count(["s3://bucket/table"])
