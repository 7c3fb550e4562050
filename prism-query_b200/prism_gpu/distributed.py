"""Multi-GPU execution: one process per GPU over torch.distributed.

The path shards without a data-path collective except one exchange step:

* Aggregation follows the reference's distributed aggregation
  (native/prism-bench/src/handler.rs:270-344): the input rows are split into
  contiguous shards in rank order; every rank aggregates its shard on its own
  GPU under the worker config (expand_worker_aggregates: AVG -> SUM + COUNT);
  the partial tables are exchanged by one all-gather and merged on the GPU by
  the reducer's rule (hash aggregation of the partials with SUM / MIN / MAX,
  then the original aggregates rebuilt). Between GPUs the exchange is one
  NCCL all-gather of packed device buffers (prism_batch_pack /
  prism_batch_unpack), so partial tables never leave HBM; over gloo (the CPU
  tests) it is an all-gather of the same packed format built on the host
  (prism_arrow_pack / prism_arrow_unpack). The partials are merged in
  the reducer's order (its own first, then the others in rank order), the
  same on every rank, so every rank returns the reducer's result.
* Joins: the build side is broadcast in the packed format (one NCCL
  broadcast of the device buffer; every rank holds a replica in HBM) and each
  rank probes its own probe shard; the shards' outputs concatenated in rank
  order are the single-GPU output.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import pyarrow as pa

from .config import HashAggConfig


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [begin, end) rows of `rank` among `world` (first ranks take the remainder)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    q, r = divmod(n, world)
    begin = rank * q + min(rank, r)
    return begin, begin + q + (1 if rank < r else 0)


def shard_batches(batches: Sequence[pa.RecordBatch], rank: int, world: int) -> List[pa.RecordBatch]:
    """The rows of `rank`'s shard of the concatenated batches, as slices (no copy)."""
    total = sum(b.num_rows for b in batches)
    begin, end = shard_range(total, rank, world)
    out, pos = [], 0
    for b in batches:
        lo, hi = max(begin, pos), min(end, pos + b.num_rows)
        if lo < hi:
            out.append(b.slice(lo - pos, hi - lo))
        pos += b.num_rows
    if not out and batches:
        out.append(batches[0].slice(0, 0))
    return out


def reducer_order(world: int, reducer: int = 0) -> List[int]:
    """Ranks in the order the reducer merges their partials: its own first,
    then its peers by index (handler.rs:314-319)."""
    if not 0 <= reducer < world:
        raise ValueError("reducer out of range")
    return [reducer] + [r for r in range(world) if r != reducer]


def _gather_bytes(data: bytes, group=None) -> List[bytes]:
    """Every rank's bytes, in rank order, over a host (gloo) group: the sizes
    are all-gathered, every buffer is padded to the largest and one
    all-gather moves them (the same steps as the device exchange)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([len(data)], dtype=torch.int64), group=group)
    host_sizes = [int(x.item()) for x in sizes]
    cap = max(max(host_sizes), 1)
    send = torch.zeros(cap, dtype=torch.uint8)
    if data:
        send[: len(data)] = torch.frombuffer(bytearray(data), dtype=torch.uint8)
    recv = [torch.empty(cap, dtype=torch.uint8) for _ in range(world)]
    dist.all_gather(recv, send, group=group)
    return [recv[r][: host_sizes[r]].numpy().tobytes() for r in range(world)]


def all_gather_batches(batch: pa.RecordBatch, group=None) -> List[pa.RecordBatch]:
    """Every rank's batch, in rank order, over a host (gloo) group: each rank
    packs its batch in the library's exchange format (prism_arrow_pack), the
    packed buffers are all-gathered, and each piece is unpacked
    (prism_arrow_unpack)."""
    from . import pack_arrow, unpack_arrow

    return [unpack_arrow(b) for b in _gather_bytes(bytes(pack_arrow(batch)), group)]


def all_gather_device_batches(batch, group=None) -> list:
    """Every rank's device batch, in rank order, as device batches on this
    rank's GPU: the batch is packed into one device buffer, the packed sizes
    are all-gathered, every buffer is padded to the largest and one
    all-gather moves them (NCCL over NVLink); each rank's piece is unpacked."""
    import torch
    import torch.distributed as dist

    from . import DeviceBatch

    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device())
    size = batch.packed_size()
    sizes = torch.zeros(world, dtype=torch.int64, device=dev)
    dist.all_gather_into_tensor(sizes, torch.tensor([size], dtype=torch.int64, device=dev), group=group)
    host_sizes = [int(x) for x in sizes.tolist()]
    cap = max(host_sizes)  # packed sizes are multiples of 16: every piece stays aligned
    send = torch.empty(cap, dtype=torch.uint8, device=dev)
    batch.pack_into(send.data_ptr(), cap)
    batch.ctx.synchronize()
    recv = torch.empty(world * cap, dtype=torch.uint8, device=dev)
    dist.all_gather_into_tensor(recv, send, group=group)
    torch.cuda.current_stream().synchronize()
    return [DeviceBatch.unpack(recv.data_ptr() + r * cap, host_sizes[r], ctx=batch.ctx) for r in range(world)]


def gather_partials(part, group=None, reducer: int = 0) -> list:
    """Every rank's partial aggregate in the reducer's merge order: device
    batches over an NCCL group, Arrow batches otherwise."""
    import torch.distributed as dist

    from . import DeviceBatch

    world = dist.get_world_size(group)
    if isinstance(part, DeviceBatch) and dist.get_backend(group) == "nccl":
        every = all_gather_device_batches(part, group)
    else:
        every = all_gather_batches(part.to_arrow() if isinstance(part, DeviceBatch) else part, group)
    return [every[r] for r in reducer_order(world, reducer)]


def broadcast_batch(batch, src: int = 0, group=None, ctx=None):
    """`src`'s batch on every rank (the build side of a sharded join,
    replacing the concatenated build broadcast of
    prism-substrait/src/executor.rs:222-232).

    Over an NCCL group the batch travels in HBM: `src` packs it into one
    device buffer (prism_batch_pack; a host batch is imported first), the
    packed size and then the buffer go out in one broadcast each, and every
    rank unpacks its copy (prism_batch_unpack); the result is a DeviceBatch.
    Over a host (gloo) group the packed bytes are built and read on the host
    (prism_arrow_pack / prism_arrow_unpack); the result is a host batch."""
    import torch
    import torch.distributed as dist

    from . import DeviceBatch, default_context, pack_arrow, unpack_arrow

    me = dist.get_rank(group)
    if dist.get_backend(group) == "nccl":
        ctx = ctx or default_context()
        dev = torch.device("cuda", torch.cuda.current_device())
        size = torch.zeros(1, dtype=torch.int64, device=dev)
        db = None
        if me == src:
            db = batch if isinstance(batch, DeviceBatch) else DeviceBatch.from_arrow(batch, ctx)
            size.fill_(db.packed_size())
        dist.broadcast(size, src=src, group=group)
        n = int(size.item())
        buf = torch.empty(max(n, 16), dtype=torch.uint8, device=dev)
        if me == src:
            db.pack_into(buf.data_ptr(), buf.numel())
            db.ctx.synchronize()
        dist.broadcast(buf, src=src, group=group)
        torch.cuda.current_stream().synchronize()
        return DeviceBatch.unpack(buf.data_ptr(), n, ctx=ctx)
    data = bytes(pack_arrow(batch)) if me == src else b""
    size = torch.tensor([len(data)], dtype=torch.int64)
    dist.broadcast(size, src=src, group=group)
    buf = torch.zeros(max(int(size.item()), 1), dtype=torch.uint8)
    if me == src and data:
        buf[: len(data)] = torch.frombuffer(bytearray(data), dtype=torch.uint8)
    dist.broadcast(buf, src=src, group=group)
    return unpack_arrow(buf[: int(size.item())].numpy().tobytes())


def _merge(parts, cfg: HashAggConfig, merge: Optional[Callable], kw) -> pa.RecordBatch:
    if merge:
        return merge(parts, cfg)
    from . import merge_partial_aggregates

    return merge_partial_aggregates(parts, cfg, **kw)


def sharded_hash_aggregate(local_batches: Sequence, cfg: HashAggConfig, group=None, local: Optional[Callable] = None,
                           merge: Optional[Callable] = None, reducer: int = 0, **kw) -> pa.RecordBatch:
    """hash_aggregate_batches over the union of every rank's shard, as the
    reference's distributed aggregation computes it.

    local(batches, worker_cfg) computes this rank's partial table (default:
    this package's GPU hash_aggregate_batches, kept in device memory);
    merge(partials, cfg) merges them (default: the GPU merge). Keyword
    arguments such as `ctx` are passed on to the defaults.
    """
    from . import expand_worker_aggregates, hash_aggregate_batches

    wcfg = expand_worker_aggregates(cfg)
    part = local(local_batches, wcfg) if local else hash_aggregate_batches(local_batches, wcfg, as_device=True, **kw)
    return _merge(gather_partials(part, group, reducer), cfg, merge, kw)


def sharded_filter_project_aggregate(local_batches: Sequence, predicate, column_indices, expressions,
                                     cfg: HashAggConfig, group=None, local: Optional[Callable] = None,
                                     merge: Optional[Callable] = None, reducer: int = 0, **kw) -> pa.RecordBatch:
    """filter_project_aggregate over the union of every rank's shard."""
    from . import expand_worker_aggregates, filter_project_aggregate

    wcfg = expand_worker_aggregates(cfg)
    if local:
        part = local(local_batches, predicate, column_indices, expressions, wcfg)
    else:
        part = filter_project_aggregate(local_batches, predicate, column_indices, expressions, wcfg,
                                        as_device=True, **kw)
    return _merge(gather_partials(part, group, reducer), cfg, merge, kw)


def sharded_join_aggregate(local_probes: Sequence, build: Optional[pa.RecordBatch], probe_keys, build_keys,
                           column_indices, expressions, cfg: HashAggConfig, group=None, src: int = 0,
                           local: Optional[Callable] = None, merge: Optional[Callable] = None, reducer: int = 0,
                           **kw) -> pa.RecordBatch:
    """join_aggregate with the build side broadcast from `src` and the probe
    rows sharded: partial aggregates per rank, merged after one all-gather
    (prism-substrait/src/executor.rs:333-842 on each worker)."""
    from . import expand_worker_aggregates, join_aggregate

    build = broadcast_batch(build, src=src, group=group)
    wcfg = expand_worker_aggregates(cfg)
    if local:
        part = local(local_probes, build, probe_keys, build_keys, column_indices, expressions, wcfg)
    else:
        part = join_aggregate(local_probes, build, probe_keys, build_keys, column_indices, expressions, wcfg,
                              as_device=True, **kw)
    return _merge(gather_partials(part, group, reducer), cfg, merge, kw)


def sharded_hash_join(local_probe: pa.RecordBatch, build: Optional[pa.RecordBatch], config, group=None, src: int = 0,
                      local: Optional[Callable] = None, **kw) -> pa.RecordBatch:
    """This rank's rows of hash_join: the build side broadcast from `src`,
    joined with this rank's probe shard. For Inner, LeftSemi and LeftAnti the
    rank-ordered concatenation of the results is the single-GPU result; for
    Left each shard's unmatched probe rows follow that shard's matches, so the
    union equals the single-GPU result as a multiset. Right and Full joins
    need every probe row against each build row and are rejected."""
    from . import hash_join
    from .config import JoinType

    if config.join_type in (JoinType.Right, JoinType.Full):
        raise ValueError("Right and Full joins cannot be sharded by probe rows")

    build = broadcast_batch(build, src=src, group=group)
    return local(local_probe, build, config) if local else hash_join(local_probe, build, config, **kw)
