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


@pytest.mark.parametrize("mode", ["1", "0"])
def test_unique_int64_keys_dense_and_hash_tables(ctx, mode, monkeypatch):
    """Unique Int64 build keys over a compact range use the dense table
    (PRISM_JOIN_DENSE unset or 1); the hash table (0) must give the same rows.
    A repeated key in a compact range falls back to the hash table."""
    monkeypatch.setenv("PRISM_JOIN_DENSE", mode)
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
