"""The per-shape tuning table (no GPU): records load from and save to the
text format, bad records are rejected with InvalidArgument, and loading a
file merges its records into the table."""
import os

import pytest

import prism_gpu


@pytest.fixture(autouse=True)
def clean_table():
    prism_gpu.tuning_clear()
    yield
    prism_gpu.tuning_clear()


def test_round_trip(tmp_path):
    p = tmp_path / "tune.txt"
    p.write_text("# comment\n"
                 "join kind=0 build=23 dense=0 lf=0.7 part=1 bits=6\n"
                 "join kind=1 build=24 dense=0 lf=0.5 part=0 bits=8\n"
                 "join_agg kind=1 build=24 block=512 blocks=3 rows=2 table=9\n"
                 "agg rows=20 block=512\n")
    prism_gpu.tuning_load(str(p))
    dump = prism_gpu.tuning_dump()
    for line in p.read_text().splitlines()[1:]:
        assert line in dump
    q = tmp_path / "again.txt"
    prism_gpu.tuning_save(str(q))
    prism_gpu.tuning_clear()
    assert "join " not in prism_gpu.tuning_dump()
    prism_gpu.tuning_load(str(q))
    assert prism_gpu.tuning_dump() == dump


@pytest.mark.parametrize("line", [
    "join kind=0 build=23 dense=0 lf=0.7 part=2 bits=6",   # partition flag out of range
    "join kind=0 build=23 dense=0 lf=0.7 part=1 bits=9",   # fan-out beyond 2^8
    "join_agg kind=1 build=24 block=300 blocks=3 rows=2 table=9",
    "join_agg kind=1 build=24 block=512 blocks=3 rows=3 table=9",
    "agg rows=20 block=100",
    "join kind=0 build=23 dense=0",                          # missing fields
    "sort rows=3",                                           # unknown record
    "join kind=0 build=23 dense=0 lf=0.7 part=1 bits",     # not key=value
])
def test_bad_records_are_rejected(tmp_path, line):
    p = tmp_path / "bad.txt"
    p.write_text(line + "\n")
    with pytest.raises(prism_gpu.PrismError) as e:
        prism_gpu.tuning_load(str(p))
    assert e.value.kind == "InvalidArgument"
    assert "join" not in prism_gpu.tuning_dump().split("\n", 1)[1]  # nothing half-loaded


def test_missing_file_is_an_error(tmp_path):
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.tuning_load(str(tmp_path / "absent.txt"))
    with pytest.raises(prism_gpu.PrismError):
        prism_gpu.tuning_save(os.path.join(str(tmp_path), "no-such-dir", "t.txt"))
