"""Multi-rank host logic on CPU: two gloo ranks shard the rows, compute their
partial tables under the reference's worker config (with the oracle standing
in for each rank's GPU), exchange them through the library's own exchange
(each partial packed by prism_arrow_pack in the format prism_batch_pack
writes on a GPU, the packed sizes and buffers all-gathered, each piece
unpacked by prism_arrow_unpack; the join build side broadcast the same way),
and merge them by the reference's reducer rule (the oracle's restatement of
prism-bench/src/handler.rs:327-344).
The merged result must reproduce the single-call result of the oracle — same
groups in the same first-seen order, integer results exact, Float64 within
1e-12 — where the decomposition is exact (no COUNT DISTINCT, no group whose
values are all null on one rank). Joins: the build side is broadcast and the
probe sharded; the rank-ordered concatenation must equal the single-call
join."""
import json
import os
import sys

import numpy as np
import pyarrow as pa
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORLD = 2


def _data(seed=7, n=60_000, nb=3):
    rng = np.random.default_rng(seed)
    out = []
    for b in range(nb):
        k = rng.integers(-3, 40, n)
        out.append(pa.RecordBatch.from_arrays([
            pa.array(k, mask=rng.random(n) < 0.02),
            pa.array(rng.integers(-10**6, 10**6, n), mask=rng.random(n) < 0.05),
            pa.array(rng.normal(0, 5, n)),
            pa.DictionaryArray.from_arrays(pa.array(rng.integers(0, 3, n).astype(np.int8)), pa.array(["A", "N", "R"])),
            pa.array(rng.integers(0, 2526, n).astype(np.int32)),
        ], names=["k", "vi", "vf", "flag", "day"]))
    return out


def _join_data(seed=9):
    rng = np.random.default_rng(seed)
    nb = 5000
    build = pa.RecordBatch.from_arrays([pa.array(rng.permutation(nb).astype(np.int64)),
                                        pa.array(rng.integers(0, 25, nb).astype(np.int32))], names=["key", "gid"])
    probes = []
    for s in range(3):
        r = np.random.default_rng(seed + 1 + s)
        probes.append(pa.RecordBatch.from_arrays([pa.array(r.integers(-100, nb + 500, 20_000)),
                                                  pa.array(r.lognormal(5, 1, 20_000))], names=["key", "amount"]))
    return build, probes


def _rank_main(rank, world, store, outdir):
    for p in (os.path.join(ROOT, "prism-query_b200"), os.path.join(ROOT, "tests"), ROOT):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import oracle_py as oracle
    from helpers import assert_batches_equal
    from prism_gpu import AggExpr, AggFunc, HashAggConfig, HashJoinConfig, JoinType, Predicate, ScalarValue
    from prism_gpu import distributed as D

    dist.init_process_group("gloo", init_method=f"file://{store}", rank=rank, world_size=world)
    try:
        data = _data()
        mine = D.shard_batches(data, rank, world)
        F = AggFunc
        # grouped: int key with nulls (null and 0 share a group, as in the reference)
        cfg = HashAggConfig([0], [AggExpr(1, F.Sum, "s"), AggExpr(1, F.Count, "n"), AggExpr(2, F.Avg, "a"),
                                  AggExpr(1, F.Min, "mn"), AggExpr(2, F.Max, "mx"), AggExpr(2, F.Sum, "sf")])
        local = lambda b, c: oracle.hash_aggregate_batches(b, c, n_threads=1)  # noqa: E731
        merge = lambda p, c: oracle.merge_partial_aggregates(p, c, n_threads=1)  # noqa: E731
        got = D.sharded_hash_aggregate(mine, cfg, local=local, merge=merge)
        ref = oracle.hash_aggregate_batches(data, cfg, n_threads=1)
        assert_batches_equal(got, ref, float_cols=(1, 3, 4, 5, 6))
        # reducer 1 merges its own partial first: its groups lead
        got1 = D.sharded_hash_aggregate(mine, cfg, local=local, merge=merge, reducer=1)
        wcfg, _ = oracle.expand_worker_aggregates(cfg)
        shards = [oracle.hash_aggregate_batches(D.shard_batches(data, r, world), wcfg, n_threads=1) for r in (1, 0)]
        assert_batches_equal(got1, oracle.merge_partial_aggregates(shards, cfg, n_threads=1), float_cols=(1, 3, 4, 5, 6))
        # global (no GROUP BY): nulls skipped
        gcfg = HashAggConfig([], [AggExpr(1, F.Sum, "s"), AggExpr(1, F.Count, "n"), AggExpr(1, F.Avg, "a"),
                                  AggExpr(1, F.Min, "mn"), AggExpr(2, F.Max, "mx")])
        got = D.sharded_hash_aggregate(mine, gcfg, local=local, merge=merge)
        ref = oracle.hash_aggregate_batches(data, gcfg, n_threads=1)
        assert_batches_equal(got, ref, float_cols=(0, 2, 3, 4))
        # fused filter -> project -> aggregate, GROUP BY a dictionary column
        pred = Predicate.Le(4, ScalarValue.Int32(2000))
        fcfg = HashAggConfig([0], [AggExpr(1, F.Sum, "s"), AggExpr(2, F.Avg, "a"), AggExpr(1, F.Count, "n")])
        got = D.sharded_filter_project_aggregate(
            mine, pred, [3, 1, 2], [], fcfg, merge=merge,
            local=lambda b, p, c, e, g: oracle.filter_project_aggregate(b, p, c, e, g, n_threads=1))
        ref = oracle.filter_project_aggregate(data, pred, [3, 1, 2], [], fcfg, n_threads=1)
        assert_batches_equal(got, ref, float_cols=(1, 2))
        # join -> aggregate: build broadcast from rank 0, probe sharded
        build, probes = _join_data()
        jcfg = HashAggConfig([0], [AggExpr(1, F.Sum, "s"), AggExpr(1, F.Count, "n")])
        got = D.sharded_join_aggregate(D.shard_batches(probes, rank, world), build if rank == 0 else None, [0], [0],
                                       [3, 1], [], jcfg, merge=merge,
                                       local=lambda p, b, pk, bk, c, e, g: oracle.join_aggregate(p, b, pk, bk, c, e, g, n_threads=1))
        ref = oracle.join_aggregate(probes, build, [0], [0], [3, 1], [], jcfg, n_threads=1)
        assert_batches_equal(got, ref, float_cols=(1,))
        # join: rank-ordered concatenation of the shards' results
        pall = pa.Table.from_batches(probes).combine_chunks().to_batches()[0]
        for jt in (JoinType.Inner, JoinType.Left, JoinType.LeftAnti):
            jc = HashJoinConfig(jt, build_keys=[0], probe_keys=[0])
            b0, b1 = D.shard_range(pall.num_rows, rank, world)
            part = D.sharded_hash_join(pall.slice(b0, b1 - b0), build if rank == 0 else None, jc,
                                       local=lambda p, b, c: oracle.hash_join(p, b, c, n_threads=1))
            every = D.all_gather_batches(part)
            got = pa.Table.from_batches(every).combine_chunks()
            ref = pa.Table.from_batches([oracle.hash_join(pall, build, jc, n_threads=1)])
            if jt == JoinType.Left:  # unmatched rows trail each shard: compare as multisets
                keys = [(n, "ascending") for n in ref.schema.names]
                got, ref = got.sort_by(keys), ref.sort_by(keys)
            assert_batches_equal(got.combine_chunks().to_batches()[0], ref.combine_chunks().to_batches()[0])
        # the exchange itself: every rank's packed batch comes back bit-exact
        # (nulls, a sliced Utf8 column, dictionaries) in rank order
        b = data[rank].slice(11 * rank + 3, 5_000)
        every = D.all_gather_batches(b)
        for r in range(world):
            assert every[r].equals(data[r].slice(11 * r + 3, 5_000))
        bb = D.broadcast_batch(build if rank == 1 else None, src=1)
        assert bb.equals(build)
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"ok": True}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_merge_partials_and_shard_joins(tmp_path):
    # a file store for the rendezvous: no port to race for
    mp.spawn(_rank_main, args=(WORLD, str(tmp_path / "pg_store"), str(tmp_path)), nprocs=WORLD, join=True)
    for r in range(WORLD):
        assert json.load(open(tmp_path / f"rank{r}.json"))["ok"]


def test_shard_ranges_cover_rows_once():
    from prism_gpu.distributed import shard_range

    for n in (0, 1, 7, 100):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
