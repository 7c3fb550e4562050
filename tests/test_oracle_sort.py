"""The oracle's sort (sort.rs restated) against an independent engine:
pyarrow's stable sort_indices with the same keys, on seeded data with nulls,
NaN, signed zeros, ties, Utf8 and dictionary keys, plus the reference's
known answers of sort.rs's own tests (sort.rs:255-299)."""
import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

import oracle_py as oracle
from prism_gpu import NullOrdering as N
from prism_gpu import SortDirection as D
from prism_gpu import SortKey


def table(n, seed):
    rng = np.random.default_rng(seed)
    f = rng.normal(0, 10, n).round(1)
    f[rng.random(n) < 0.03] = np.nan
    f[rng.random(n) < 0.03] = -0.0
    f[rng.random(n) < 0.03] = 0.0
    return pa.RecordBatch.from_arrays(
        [pa.array(rng.integers(-5, 5, n), mask=rng.random(n) < 0.1),
         pa.array(f, mask=rng.random(n) < 0.05),
         pa.array(np.array(["b", "a", "ab", "", "ba", "a\x00"])[rng.integers(0, 6, n)], mask=rng.random(n) < 0.05),
         pa.array(rng.integers(0, 3, n).astype(np.int32)),
         pa.array(np.arange(n))],
        names=["i", "f", "s", "g", "row"])


def arrow_order(batch, keys):
    """pyarrow's stable sort, with floats by totalOrder (pyarrow orders NaN
    last and -0.0 == +0.0, so floats are sorted through their totalOrder key)."""
    cols, spec = [], []
    for j, k in enumerate(keys):
        c = batch.column(k.column)
        if pa.types.is_floating(c.type):
            bits = np.frombuffer(np.asarray(c.to_numpy(zero_copy_only=False), dtype=np.float64).tobytes(), dtype=np.int64)
            tk = bits ^ ((bits >> 63).astype(np.uint64) >> np.uint64(1)).astype(np.int64)
            c = pa.array(tk, mask=np.asarray(c.is_null()))
        cols.append(c)
        spec.append((f"k{j}", "descending" if k.direction == D.Desc else "ascending"))
    t = pa.table(cols, names=[f"k{j}" for j in range(len(keys))])
    # null placement per key: pyarrow has one null_placement for all keys
    placements = {k.nulls for k in keys}
    assert len(placements) == 1
    np_ = "at_start" if keys[0].nulls == N.NullsFirst else "at_end"
    return pc.sort_indices(t, sort_keys=spec, null_placement=np_).to_numpy()


@pytest.mark.parametrize("nulls", [N.NullsFirst, N.NullsLast])
@pytest.mark.parametrize("spec", [[(0, D.Asc)], [(1, D.Desc)], [(2, D.Asc)], [(3, D.Desc), (1, D.Asc)],
                                  [(2, D.Desc), (0, D.Asc), (1, D.Desc)]])
def test_oracle_sort_matches_pyarrow(spec, nulls):
    b = table(3_000, 7)
    keys = [SortKey(c, d, nulls) for c, d in spec]
    got = oracle.sort_batch(b, keys)
    assert got.column(4).to_numpy().tolist() == arrow_order(b, keys).tolist()


def test_oracle_sort_limit_and_edges():
    b = table(500, 3)
    keys = [SortKey(1, D.Desc, N.NullsLast)]
    full = oracle.sort_batch(b, keys)
    top = oracle.sort_batch(b, keys, limit=10)
    assert top.num_rows == 10 and top.column(4).equals(full.column(4).slice(0, 10))
    assert oracle.sort_batch(b, []).column(4).equals(b.column(4))  # unchanged (NaN keeps .equals from holding)
    assert oracle.sort_batch(b.slice(0, 0), keys).num_rows == 0
    with pytest.raises(oracle.OracleError):
        oracle.sort_batch(b, [SortKey(9)])


def test_reference_known_answers():
    """sort.rs's own tests (sort.rs:255-299)."""
    from golden import reference_kat as K

    b = K.sort_test_batch()
    names = oracle.sort_batch(b, K.SORT_BY_NAME_ASC).column(0).to_pylist()
    assert names[0] == "Alice" and names[4] == "Eve"
    top = oracle.sort_batch(b, K.SORT_BY_SCORE_DESC, limit=3)
    assert top.num_rows == 3 and top.column(2)[0].as_py() == 92.0
    multi = oracle.sort_batch(b, K.SORT_MULTI_KEY)
    assert multi.column(1)[0].as_py() == 25 and multi.column(2)[0].as_py() == 92.0
