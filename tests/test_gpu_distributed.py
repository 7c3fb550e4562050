"""The multi-GPU exchange step on one GPU: device batches packed into one
device buffer and unpacked (every column type, nulls, slices, empty), the
reducer merge of partial aggregates on the GPU against the oracle's
restatement of prism-bench/src/handler.rs:327-344 (its own known answers,
then partials of 4 shards laid out as one all-gather lays them out), and
the whole path through a real NCCL process group of one rank."""
import numpy as np
import pyarrow as pa
import pytest

import oracle_py as oracle
import prism_gpu
from golden import reference_kat as K
from helpers import assert_batches_equal
from prism_gpu import AggExpr, AggFunc, DeviceBatch, HashAggConfig, HashJoinConfig, JoinType
from prism_gpu import distributed as D

pytestmark = pytest.mark.gpu
F = AggFunc


def _typed_batch(n, seed):
    rng = np.random.default_rng(seed)
    words = np.array(["", "a", "bb", "ccc", "delta", "epsilon-long-value", "z" * 40])
    dec = [None if rng.random() < 0.1 else int(v) for v in rng.integers(-10**12, 10**12, n)]
    return pa.RecordBatch.from_arrays([
        pa.array(rng.integers(-100, 100, n), mask=rng.random(n) < 0.1),
        pa.array(rng.normal(0, 1, n), mask=rng.random(n) < 0.05),
        pa.array(words[rng.integers(0, len(words), n)], mask=rng.random(n) < 0.1),
        pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 3, n).astype(np.int8)), pa.array(["x", "yy", "zzz"])),
        pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.1),
        pa.array(rng.integers(0, 20000, n).astype(np.int32), type=pa.date32()),
        pa.array(dec, type=pa.decimal128(18, 3)),
        pa.array(rng.integers(0, 255, n).astype(np.uint8)),
        pa.array(rng.integers(-5, 5, n).astype(np.int32)),
    ], names=["i64", "f64", "s", "d", "b", "day", "dec", "u8", "i32"])


def _pack_all(parts):
    """Packs device batches at r * cap of one device buffer, as an all-gather
    of padded buffers leaves them; returns the buffer, cap and sizes."""
    import torch

    sizes = [p.packed_size() for p in parts]
    assert all(s % 16 == 0 for s in sizes)
    cap = max(sizes)
    buf = torch.empty(len(parts) * cap, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    for r, p in enumerate(parts):
        p.pack_into(buf.data_ptr() + r * cap, cap)
    return buf, cap, sizes


@pytest.mark.parametrize("rows,offset", [(5000, 0), (3000, 777), (0, 0), (1, 0)])
def test_pack_round_trip(ctx, rows, offset):
    b = _typed_batch(rows + offset, 3).slice(offset, rows)
    d = DeviceBatch.from_arrow(b, ctx)
    buf, cap, sizes = _pack_all([d, d])
    ctx.synchronize()
    want = d.to_arrow()
    assert want.to_pylist() == b.to_pylist()
    for r in range(2):
        back = DeviceBatch.unpack(buf.data_ptr() + r * cap, sizes[r], ctx).to_arrow()
        assert back.schema == want.schema
        assert back.equals(want)


def test_unpack_rejects_bad_headers(ctx):
    import torch

    d = DeviceBatch.from_arrow(_typed_batch(100, 1), ctx)
    size = d.packed_size()
    buf = torch.zeros(size, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(prism_gpu.PrismError):  # no magic word
        DeviceBatch.unpack(buf.data_ptr(), size, ctx)
    d.pack_into(buf.data_ptr(), size)
    ctx.synchronize()
    with pytest.raises(prism_gpu.PrismError):  # shorter than the packed batch
        DeviceBatch.unpack(buf.data_ptr(), size - 16, ctx)
    with pytest.raises(prism_gpu.PrismError):  # destination too small
        d.pack_into(buf.data_ptr(), size - 16)
    assert DeviceBatch.unpack(buf.data_ptr(), size, ctx).num_rows == 100


def test_reducer_known_answers(ctx):
    """handler.rs:1378-1460 on the GPU."""
    got = prism_gpu.merge_partial_aggregates(K.partial_batches(), K.MERGE_ORIGINAL, ctx=ctx)
    ref = oracle.merge_partial_aggregates(K.partial_batches(), K.MERGE_ORIGINAL)
    assert_batches_equal(got, ref, float_cols=(1, 3))
    rows = {r["status"]: (r["agg_0"], r["agg_1"], r["agg_2"]) for r in got.to_pylist()}
    assert rows == K.MERGE_EXPECTED


def _merge_data(n=400_000, seed=11):
    rng = np.random.default_rng(seed)
    key = rng.integers(0, 300, n)
    v = rng.integers(-10**6, 10**6, n)
    vmask = rng.random(n) < 0.05
    vmask[key == 7] = True  # group 7: every value null
    vmask[(key == 8) & (np.arange(n) >= n // 2)] = True  # group 8: null in the later shards only
    names = np.array([f"cust-{i:04d}" for i in range(500)])
    return [pa.RecordBatch.from_arrays([
        pa.array(key, mask=rng.random(n) < 0.01),
        pa.array(v, mask=vmask),
        pa.array(rng.lognormal(3, 1, n)),
        pa.array(names[rng.integers(0, 500, n)]),
        pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 3, n).astype(np.int8)), pa.array(["A", "N", "R"])),
    ], names=["k", "v", "x", "cust", "flag"])]


AGG_CASES = {
    "int_key_all_funcs": HashAggConfig([0], [AggExpr(1, F.Sum, "s"), AggExpr(1, F.Count, "n"), AggExpr(2, F.Avg, "a"),
                                            AggExpr(1, F.Min, "mn"), AggExpr(2, F.Max, "mx"),
                                            AggExpr(3, F.CountDistinct, "cd")]),
    "utf8_key": HashAggConfig([3], [AggExpr(2, F.Sum, "s"), AggExpr(1, F.Avg, "a"), AggExpr(1, F.Count, "n")]),
    "two_keys": HashAggConfig([4, 0], [AggExpr(2, F.Avg, "a"), AggExpr(1, F.Max, "mx")]),
    # TPC-H Q1's shape: 8 aggregates, 10 worker columns, one distinct column each in the merge
    "q1_shape": HashAggConfig([4], [AggExpr(2, F.Sum, "sum_x"), AggExpr(1, F.Sum, "sum_v"), AggExpr(2, F.Avg, "avg_x"),
                                    AggExpr(1, F.Avg, "avg_v"), AggExpr(1, F.Count, "n"), AggExpr(2, F.Min, "mn"),
                                    AggExpr(1, F.Max, "mx"), AggExpr(3, F.CountDistinct, "cd")]),
    "global": HashAggConfig([], [AggExpr(1, F.Sum, "s"), AggExpr(1, F.Avg, "a"), AggExpr(2, F.Min, "mn"),
                                 AggExpr(1, F.Count, "n")]),
}


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("name", sorted(AGG_CASES))
def test_sharded_merge_matches_reducer(ctx, name, world):
    """World partials computed on the GPU, packed as an all-gather leaves
    them, unpacked and merged on the GPU: the oracle reducer's result over
    the oracle's partials (bit-exact keys and counts, Float64 within 1e-12)."""
    cfg = AGG_CASES[name]
    data = _merge_data()
    wcfg = prism_gpu.expand_worker_aggregates(cfg)
    parts = [prism_gpu.hash_aggregate_batches(D.shard_batches(data, r, world), wcfg, ctx=ctx, as_device=True)
             for r in range(world)]
    buf, cap, sizes = _pack_all(parts)
    ctx.synchronize()
    got_parts = [DeviceBatch.unpack(buf.data_ptr() + r * cap, sizes[r], ctx) for r in range(world)]
    got = prism_gpu.merge_partial_aggregates(got_parts, cfg, ctx=ctx)
    ocfg, _ = oracle.expand_worker_aggregates(cfg)
    ref_parts = [oracle.hash_aggregate_batches(D.shard_batches(data, r, world), ocfg) for r in range(world)]
    for g, o in zip(got_parts, ref_parts):
        assert_batches_equal(g.to_arrow(), o, float_cols=tuple(range(g.num_columns)))
    ref = oracle.merge_partial_aggregates(ref_parts, cfg)
    nk = len(cfg.group_by)
    floats = tuple(nk + i for i, a in enumerate(cfg.aggregates) if a.func in (F.Sum, F.Avg, F.Min, F.Max))
    assert_batches_equal(got, ref, float_cols=floats)


def test_reducer_order(ctx):
    """Reducer 2 of 3 merges its own partial first: its groups lead."""
    cfg = AGG_CASES["utf8_key"]
    data = _merge_data(n=30_000, seed=5)
    wcfg = prism_gpu.expand_worker_aggregates(cfg)
    parts = [prism_gpu.hash_aggregate_batches(D.shard_batches(data, r, 3), wcfg, ctx=ctx) for r in range(3)]
    order = D.reducer_order(3, 2)
    assert order == [2, 0, 1]
    got = prism_gpu.merge_partial_aggregates([parts[r] for r in order], cfg, ctx=ctx)
    ref = oracle.merge_partial_aggregates([parts[r] for r in order], cfg)
    assert_batches_equal(got, ref, float_cols=(1, 2))
    assert got.column(0)[0] == parts[2].column(0)[0]


def test_merge_errors(ctx):
    cfg = AGG_CASES["two_keys"]
    with pytest.raises(prism_gpu.PrismError):  # partial without the worker columns
        prism_gpu.merge_partial_aggregates([_merge_data(n=100)[0]], cfg, ctx=ctx)
    with pytest.raises(prism_gpu.PrismError):  # the reducer always has its own partial
        prism_gpu.merge_partial_aggregates([], AGG_CASES["utf8_key"], ctx=ctx)
    wcfg = prism_gpu.expand_worker_aggregates(AGG_CASES["utf8_key"])
    empty = [_merge_data(n=100)[0].slice(0, 0)]
    part = prism_gpu.hash_aggregate_batches(empty, wcfg, ctx=ctx)
    ocfg, _ = oracle.expand_worker_aggregates(AGG_CASES["utf8_key"])
    assert_batches_equal(part, oracle.hash_aggregate_batches(empty, ocfg))
    got = prism_gpu.merge_partial_aggregates([part, part], AGG_CASES["utf8_key"], ctx=ctx)
    assert_batches_equal(got, oracle.merge_partial_aggregates([part, part], AGG_CASES["utf8_key"]))


def test_nccl_group_of_one(ctx, tmp_path):
    """sharded_hash_aggregate through a real NCCL process group (one rank):
    the device partial is packed, all-gathered by NCCL and merged on the GPU."""
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"file://{tmp_path / 'store'}", rank=0, world_size=1)
    try:
        data = _merge_data(n=50_000, seed=2)
        for cfg in (AGG_CASES["int_key_all_funcs"], AGG_CASES["global"]):
            got = D.sharded_hash_aggregate(data, cfg, ctx=ctx)
            ocfg, _ = oracle.expand_worker_aggregates(cfg)
            ref = oracle.merge_partial_aggregates([oracle.hash_aggregate_batches(data, ocfg)], cfg)
            nk = len(cfg.group_by)
            floats = tuple(nk + i for i, a in enumerate(cfg.aggregates) if a.func in (F.Sum, F.Avg, F.Min, F.Max))
            assert_batches_equal(got, ref, float_cols=floats)
        # sharded join -> aggregate and join: the build side broadcast as one
        # packed device buffer (NCCL), unpacked into HBM
        rng = np.random.default_rng(12)
        build = pa.RecordBatch.from_arrays([pa.array(rng.permutation(4000).astype(np.int64)),
                                            pa.array(rng.integers(0, 25, 4000).astype(np.int32)),
                                            pa.array([f"b{i % 31}" for i in range(4000)])], names=["key", "gid", "tag"])
        probes = [pa.RecordBatch.from_arrays([pa.array(rng.integers(-50, 4500, 30_000)), pa.array(rng.lognormal(5, 1, 30_000))],
                                             names=["key", "amount"]) for _ in range(2)]
        jcfg = HashAggConfig([0], [AggExpr(1, F.Sum, "s"), AggExpr(1, F.Count, "n")])
        got = D.sharded_join_aggregate(probes, build, [0], [0], [3, 1], [], jcfg, ctx=ctx)
        assert_batches_equal(got, oracle.join_aggregate(probes, build, [0], [0], [3, 1], [], jcfg), float_cols=(1,))
        jc = HashJoinConfig(JoinType.Inner, build_keys=[0], probe_keys=[0])
        got = D.sharded_hash_join(probes[0], build, jc, ctx=ctx)
        assert_batches_equal(got, oracle.hash_join(probes[0], build, jc))
        bb = D.broadcast_batch(build, ctx=ctx)
        assert bb.to_arrow().equals(build)
    finally:
        dist.destroy_process_group()
