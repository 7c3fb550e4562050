"""The allocation-free probe against the allocating one, through the C ABI.

Some callers may not allocate device memory while they run — for example a
host engine that reserved its device-memory budget up front and hands every
buffer out of its own pool. prism_hash_table_probe_noalloc serves them: the
caller passes device pointers for the probe keys and for the outputs, and
the call keeps its scratch in a fixed device array of the library. Its
results must equal prism_hash_table_probe's (same matches, same order), on
consecutive calls too, since every call shares that array.
"""
import ctypes as C

import numpy as np
import pyarrow as pa
import pytest

import prism_gpu

pytestmark = pytest.mark.gpu

MAX_ROWS = 131072 * 2048  # the entry point's stated maximum probe size


def _noalloc():
    f = prism_gpu.lib().prism_hash_table_probe_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64,
                  C.POINTER(C.c_int64)]
    f.restype = C.c_int
    return f


def _inputs(dup, seed):
    rng = np.random.default_rng(seed)
    n_build, n_probe = 50_000, 400_000
    bkeys = rng.integers(0, n_build // 3, n_build) if dup else rng.permutation(n_build)
    build = pa.RecordBatch.from_arrays([pa.array(bkeys.astype(np.int64)), pa.array(np.arange(n_build, dtype=np.int64))],
                                       names=["k", "v"])
    pkeys = rng.integers(-10, int(n_build * 1.2), n_probe).astype(np.int64)
    pkeys[:5] = [np.iinfo(np.int64).min, -1, 0, 1, np.iinfo(np.int64).max]
    return build, pkeys


@pytest.mark.parametrize("dup", [False, True])
def test_noalloc_probe_equals_allocating_probe(dup):
    import torch

    ctx = prism_gpu.default_context()
    build, pkeys = _inputs(dup, seed=11 if dup else 7)
    table = prism_gpu.HashTable.build(build, [0], ctx)
    assert table.has_duplicates == dup
    probe = pa.RecordBatch.from_arrays([pa.array(pkeys)], names=["k"])
    ref_p, ref_b = table.probe(probe, [0])  # the existing, allocating entry point
    ref_p, ref_b = ref_p.to_numpy(), ref_b.to_numpy()

    keys_dev = torch.from_numpy(pkeys).to("cuda")
    cap = len(ref_p) + 64
    out_p = torch.empty(cap, dtype=torch.int32, device="cuda")
    out_b = torch.empty(cap, dtype=torch.int32, device="cuda")
    f = _noalloc()
    for _ in range(2):  # consecutive calls share the scratch array
        out_p.fill_(-7)
        out_b.fill_(-7)
        torch.cuda.synchronize()
        m = C.c_int64(-1)
        rc = f(ctx.handle, table._h, keys_dev.data_ptr(), len(pkeys), out_p.data_ptr(), out_b.data_ptr(), cap, C.byref(m))
        assert rc == 0, prism_gpu.lib().prism_last_error(ctx.handle)
        assert m.value == len(ref_p)
        got_p = out_p[: m.value].cpu().numpy().view(np.uint32)
        got_b = out_b[: m.value].cpu().numpy().view(np.uint32)
        assert np.array_equal(got_p, ref_p)
        assert np.array_equal(got_b, ref_b)


@pytest.mark.parametrize("dup", [False, True])
def test_noalloc_probe_rejects_sizes_and_short_outputs(dup):
    import torch

    ctx = prism_gpu.default_context()
    build, pkeys = _inputs(dup, seed=3)
    table = prism_gpu.HashTable.build(build, [0], ctx)
    f = _noalloc()
    keys_dev = torch.from_numpy(pkeys).to("cuda")
    out = torch.empty(16, dtype=torch.int32, device="cuda")
    m = C.c_int64(-1)
    # over the stated maximum: rejected before any device work
    rc = f(ctx.handle, table._h, keys_dev.data_ptr(), MAX_ROWS + 1, out.data_ptr(), out.data_ptr(), 16, C.byref(m))
    assert rc == 3
    assert b"maximum" in prism_gpu.lib().prism_last_error(ctx.handle)
    # too small an output: the prefix of the matches that fits (with repeated
    # keys, a probe row's matches may straddle the capacity), nothing past it,
    # the full count reported
    ref_p, ref_b = table.probe(pa.RecordBatch.from_arrays([pa.array(pkeys)], names=["k"]), [0])
    for cap in (100, 101, 1003):
        out_p = torch.full((cap + 8,), -7, dtype=torch.int32, device="cuda")
        out_b = torch.full((cap + 8,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = f(ctx.handle, table._h, keys_dev.data_ptr(), len(pkeys), out_p.data_ptr(), out_b.data_ptr(), cap, C.byref(m))
        assert rc == 3 and m.value == len(ref_p)
        assert np.array_equal(out_p[:cap].cpu().numpy().view(np.uint32), ref_p.to_numpy()[:cap])
        assert np.array_equal(out_b[:cap].cpu().numpy().view(np.uint32), ref_b.to_numpy()[:cap])
        assert (out_p[cap:].cpu().numpy() == -7).all() and (out_b[cap:].cpu().numpy() == -7).all()
