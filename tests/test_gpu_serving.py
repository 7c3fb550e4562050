"""Serving loop (the native prism_server_* ABI through prism_gpu.serving):
every request's result is the same served in the mix (coalesced with
others, on several streams, under admission, smallest job first) as run
alone; errors come back on the request's future."""
import numpy as np
import pytest

from helpers import assert_batches_equal

pytestmark = pytest.mark.gpu


def _setup(torch, prism_gpu, ctx):
    from prism_gpu import AggExpr, AggFunc, HashAggConfig, HashTable

    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    tables = {}
    for name, n in (("t0", 200_000), ("t1", 1_300_000)):
        keys = torch.randperm(n, generator=g, device=dev)
        pay = torch.randint(-(2**62), 2**62, (n,), generator=g, device=dev)
        # torch wrote them on its stream; the library reads them on the context's
        torch.cuda.synchronize()
        db = prism_gpu.DeviceBatch.from_device_buffers([("k", "l", keys.data_ptr()), ("v", "l", pay.data_ptr())], n, ctx)
        tables[name] = (HashTable.build(db, [0], ctx), n, keys, pay)
    kpool = torch.randint(0, 1_600_000, (3_000_000,), generator=g, device=dev)
    gkeys = torch.randint(-(2**40), 2**40, (64,), generator=g, device=dev)
    akey = gkeys[torch.randint(0, 64, (3_000_000,), generator=g, device=dev)]
    avi = torch.randint(-1000, 1000, (3_000_000,), generator=g, device=dev)
    avf = torch.rand(3_000_000, generator=g, device=dev, dtype=torch.float64)
    torch.cuda.synchronize()
    cfg = HashAggConfig([0], [AggExpr(1, AggFunc.Sum, "s"), AggExpr(2, AggFunc.Avg, "a"), AggExpr(1, AggFunc.Count, "n"),
                              AggExpr(2, AggFunc.Min, "mn")])
    return tables, kpool, (akey, avi, avf), cfg


def test_served_results_equal_alone(ctx):
    import torch

    import prism_gpu
    from prism_gpu import serving as S

    tables, kpool, (akey, avi, avf), cfg = _setup(torch, prism_gpu, ctx)
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(60):
        rows = int(np.exp(rng.uniform(np.log(1000), np.log(600_000))))
        off = int(rng.integers(0, 3_000_000 - rows))
        if i % 2:
            reqs.append(S.ProbeRequest("t0" if i % 4 == 1 else "t1", kpool[off:off + rows]))
        else:
            reqs.append(S.AggRequest([("k", "l", akey[off:off + rows]), ("vi", "l", avi[off:off + rows]),
                                      ("vf", "g", avf[off:off + rows])], cfg))
    torch.cuda.synchronize()
    regs = {name: S._Table(t, 1) for name, (t, *_rest) in tables.items()}
    alone, _ = S.run_plain(reqs, regs, ctx)
    # alone: probe outputs in full, for an exact comparison
    alone_rows = {}
    for i, r in enumerate(reqs):
        if isinstance(r, S.ProbeRequest):
            db = prism_gpu.DeviceBatch.from_device_buffers([("key", "l", r.keys.data_ptr())], int(r.keys.numel()), ctx)
            out = regs[r.table].table.join_project(db, [0], [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 2])
            alone_rows[i] = (out.column(0).to_numpy(), out.column(1).to_numpy())
    srv = S.Server(0, budget_bytes=64 << 20, workers=3, coalesce_rows=1 << 17, max_coalesce=16)
    for name, reg in regs.items():
        srv.register_table(name, reg.table, 1)
    futs = [srv.submit(r) for r in reqs]
    got = [f.result(timeout=300) for f in futs]
    srv.close()
    for i, (r, a, b) in enumerate(zip(reqs, alone, got)):
        if isinstance(r, S.ProbeRequest):
            assert b.matches == a
            pr, pay = alone_rows[i]
            assert np.array_equal(b.probe_rows.cpu().numpy().astype(np.uint32), pr)
            assert np.array_equal(b.payload.cpu().numpy(), pay)
        else:
            assert_batches_equal(b, a, float_cols=(1, 2, 4))


def test_global_aggregates_and_errors(ctx):
    """GROUP BY-less aggregates run alone (never coalesced) and equal the
    plain call; a probe of an unregistered table fails at submit."""
    import torch

    import prism_gpu
    from prism_gpu import AggExpr, AggFunc, HashAggConfig
    from prism_gpu import serving as S

    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(9)
    v = torch.randint(-1000, 1000, (500_000,), generator=g, device=dev)
    x = torch.rand(500_000, generator=g, device=dev, dtype=torch.float64)
    cfg = HashAggConfig([], [AggExpr(0, AggFunc.Sum, "s"), AggExpr(1, AggFunc.Avg, "a"), AggExpr(0, AggFunc.Count, "n")])
    reqs = [S.AggRequest([("v", "l", v[i * 1000:(i + 1) * 1000 + 7 * i]), ("x", "g", x[i * 1000:(i + 1) * 1000 + 7 * i])], cfg)
            for i in range(40)]
    torch.cuda.synchronize()
    alone, _ = S.run_plain(reqs, {}, ctx)
    srv = S.Server(0, workers=2, coalesce_rows=1 << 20, max_coalesce=32)
    got = [f.result(timeout=300) for f in [srv.submit(r) for r in reqs]]
    with pytest.raises(KeyError):
        srv.submit(S.ProbeRequest("missing", v[:10]))
    srv.close()
    for a, b in zip(alone, got):
        assert_batches_equal(b, a, float_cols=(0, 1))


def _sorted_probe(res):
    rows = res.probe_rows.cpu().numpy().astype(np.int64)
    pay = res.payload.cpu().numpy()
    o = np.argsort(rows, kind="stable")
    return rows[o], pay[o]


def test_device_queue_results_equal_alone(ctx):
    """Probes drained by the persistent kernel (the device work queue): dense
    and hash tables, requests of 1 row to 700K rows (ragged tiles) mixed with
    GROUP BYs on the workers; every probe's matches equal the request run
    alone, as a multiset."""
    import torch

    import prism_gpu
    from prism_gpu import serving as S

    tables, kpool, (akey, avi, avf), cfg = _setup(torch, prism_gpu, ctx)
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(21)
    n = 700_000
    sparse = torch.randperm(n, generator=g, device=dev) * 7919 + 3  # no dense table: hash slots
    pay = torch.randint(-(2**62), 2**62, (n,), generator=g, device=dev)
    torch.cuda.synchronize()  # (written on torch's stream, read on the context's)
    db = prism_gpu.DeviceBatch.from_device_buffers([("k", "l", sparse.data_ptr()), ("v", "l", pay.data_ptr())], n, ctx)
    th = prism_gpu.HashTable.build(db, [0], ctx)
    assert th.layout == "hash" and tables["t0"][0].layout == "dense"
    hkeys = sparse[torch.randint(0, n, (1_500_000,), generator=g, device=dev)]
    hkeys[::4] += 1  # misses
    regs = {name: S._Table(t, 1) for name, (t, *_rest) in tables.items()}
    regs["th"] = S._Table(th, 1)
    rng = np.random.default_rng(23)
    reqs = []
    for i in range(90):
        rows = 1 if i == 3 else int(np.exp(rng.uniform(np.log(1000), np.log(700_000))))
        if i % 3 == 0:
            off = int(rng.integers(0, 3_000_000 - rows))
            reqs.append(S.AggRequest([("k", "l", akey[off:off + rows]), ("vi", "l", avi[off:off + rows]),
                                      ("vf", "g", avf[off:off + rows])], cfg))
        elif i % 3 == 1:
            off = int(rng.integers(0, 1_500_000 - rows))
            reqs.append(S.ProbeRequest("th", hkeys[off:off + rows]))
        else:
            off = int(rng.integers(0, 3_000_000 - rows))
            reqs.append(S.ProbeRequest("t0" if i % 2 else "t1", kpool[off:off + rows]))
    torch.cuda.synchronize()
    alone = {}
    for i, r in enumerate(reqs):
        if isinstance(r, S.ProbeRequest):
            kb = prism_gpu.DeviceBatch.from_device_buffers([("key", "l", r.keys.data_ptr())], int(r.keys.numel()), ctx)
            out = regs[r.table].table.join_project(kb, [0], [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 2])
            alone[i] = (out.column(0).to_numpy().astype(np.int64), out.column(1).to_numpy())
        else:
            alone[i] = prism_gpu.hash_aggregate(
                prism_gpu.DeviceBatch.from_device_buffers([(nm, f, t.data_ptr()) for nm, f, t in r.columns],
                                                          int(r.columns[0][2].numel()), ctx), r.config, ctx=ctx)
    srv = S.Server(0, workers=2, coalesce_rows=1 << 17, max_coalesce=16, device_queue=True)
    for name, reg in regs.items():
        srv.register_table(name, reg.table, 1)
    for _ in range(2):  # twice: the second round runs on a relaunched or still-resident kernel
        futs = [srv.submit(r) for r in reqs]
        got = [f.result(timeout=300) for f in futs]
        for i, (r, b) in enumerate(zip(reqs, got)):
            if isinstance(r, S.ProbeRequest):
                rows, pay = _sorted_probe(b)
                assert b.matches == len(alone[i][0])
                assert np.array_equal(rows, alone[i][0]) and np.array_equal(pay, alone[i][1])
            else:
                assert_batches_equal(b, alone[i], float_cols=(1, 2, 4))
        import time

        time.sleep(0.05)  # long enough for the kernel's CTAs to go idle and exit
    srv.close()


def test_device_queue_bounded_wait_times_out_and_recovers(ctx):
    """A request whose descriptor never arrives: the kernel's wait for it runs
    out (a short limit here), the request fails with Timeout, and the queue
    serves the next probes correctly."""
    import torch

    import prism_gpu
    from prism_gpu import serving as S

    tables, kpool, _, _ = _setup(torch, prism_gpu, ctx)
    regs = {name: S._Table(t, 1) for name, (t, *_rest) in tables.items()}
    srv = S.Server(0, workers=1, device_queue=True, queue_wait_limit_ms=50)
    for name, reg in regs.items():
        srv.register_table(name, reg.table, 1)
    stalled = srv.inject_unready()
    with pytest.raises(prism_gpu.PrismError) as e:
        stalled.result(timeout=60)
    assert e.value.kind == "Timeout"
    keys = kpool[:250_000]
    torch.cuda.synchronize()
    got = srv.submit(S.ProbeRequest("t1", keys)).result(timeout=60)
    kb = prism_gpu.DeviceBatch.from_device_buffers([("key", "l", keys.data_ptr())], 250_000, ctx)
    out = regs["t1"].table.join_project(kb, [0], [prism_gpu.PRISM_COL_PROBE_ROW_INDEX, 2])
    rows, pay = _sorted_probe(got)
    assert np.array_equal(rows, out.column(0).to_numpy().astype(np.int64))
    assert np.array_equal(pay, out.column(1).to_numpy())
    srv.close()
