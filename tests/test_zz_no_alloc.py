"""cellato_batch_run_noalloc -- the batched run for callers that must not
allocate device memory (an application that owns all device memory through its
own pool, a latency-critical loop that cannot take cudaMalloc's implicit
synchronisation, a fixed device-memory budget).  Its work list lives in a fixed
array of the library's device memory instead of a cudaMalloc'd buffer.

Checked through the C ABI against the existing batched entry point
(cellato_batch_create + cellato_batch_launch) on two calls in a row, with
different batches -- the second smaller than the first, so that it runs over
the longer work list the first one left behind in the array.  The path is
integer bitwise work: results must be identical (tolerance: exact).  Also: a
batch over the grid or work-item limit is refused before anything runs, and so
is a call on a stream that is being captured into a CUDA graph.  This file is
collected last on purpose."""
import numpy as np
import pytest

from cellato_b200 import inputs, lib

pytestmark = pytest.mark.gpu


def batch_specs(seed, n):
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        r = int(rng.integers(0, 10))
        X = int(rng.integers(1, 6)) * 64
        Y = int(rng.integers(1, 40)) * 8
        steps = int(rng.integers(0, 30))
        specs.append((r, X, Y, steps, rng.integers(0, inputs.STATES[r], size=(Y, X), dtype=np.uint8)))
    return specs


def upload_all(oracle, specs, layout, W):
    from cellato_b200.device import DevicePlanes
    out = []
    for r, X, Y, steps, cells in specs:
        nb = inputs.PLANES[r]
        a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
        a.upload(oracle.pack(layout, W, nb, cells))
        out.append((a, b))
    return out


@pytest.mark.parametrize("layout,W", [(1, 64)])
def test_noalloc_matches_batch_on_two_calls(cuda, oracle, layout, W):
    import torch
    from cellato_b200.batch import Batch, run_noalloc
    ks = {r: [4, 6, 5, 8, 3, 4, 2, 7, 5, 3][r] for r in range(10)}
    for call, (seed, n) in enumerate(((101, 29), (202, 11))):
        specs = batch_specs(seed, n)
        ref_bufs = upload_all(oracle, specs, layout, W)
        new_bufs = upload_all(oracle, specs, layout, W)
        grids = lambda bufs: [(r, X, Y, s, a.ptrs, b.ptrs) for (r, X, Y, s, _), (a, b) in zip(specs, bufs)]
        batch = Batch(layout, W, grids(ref_bufs), ks)
        batch.launch()
        flags = run_noalloc(layout, W, grids(new_bufs), ks)
        torch.cuda.synchronize()
        for i, ((ra, rb), (na, nb_)) in enumerate(zip(ref_bufs, new_bufs)):
            assert flags[i] == batch.result_in_b(i), (call, i)
            want = (rb if batch.result_in_b(i) else ra).download()
            got = (nb_ if flags[i] else na).download()
            assert np.array_equal(got, want), (call, i, specs[i][:4])
        batch.close()


def _call(grids, ks=None, stream=0):
    import ctypes
    from cellato_b200 import lib as L_
    L = L_.load()
    n = len(grids)
    arr = (lib.BatchGrid * max(1, n))()
    for i, (rule, X, Y, steps, pa, pb) in enumerate(grids):
        arr[i].rule, arr[i].x_cells, arr[i].y_cells, arr[i].steps = rule, X, Y, steps
        for p, ptr in enumerate(pa):
            arr[i].planes_a[p] = ptr
        for p, ptr in enumerate(pb):
            arr[i].planes_b[p] = ptr
    kv, nk = lib.k_array(ks)
    flags = (ctypes.c_int * max(1, n))()
    return L.cellato_batch_run_noalloc(1, 64, arr, n, kv, nk, stream, flags)


def test_noalloc_rejects_batches_beyond_its_limits(cuda):
    import torch
    from cellato_b200.device import DevicePlanes
    L = lib.load()
    # more grids than CELLATO_NOALLOC_MAX_GRIDS (the count is checked first)
    assert _call([(0, 64, 8, 1, [16], [32])] * 1025) == lib.EINVAL
    assert b"no-allocation limit" in L.cellato_last_error()
    # under the grid limit but over CELLATO_NOALLOC_MAX_ITEMS work items: a
    # 4096^2 WireWorld grid (two planes: tiles of 30 words x 128 rows, k = 2)
    # is 160 tiles a round, 500 rounds = 80,000 items; nothing may run
    X = Y = 4096
    wire = lib.rule_id("wire")
    a, b = DevicePlanes(2, X, Y), DevicePlanes(2, X, Y)
    a.buf.fill_(0x5A)
    torch.cuda.synchronize()
    rc = _call([(wire, X, Y, 1000, a.ptrs, b.ptrs)], {wire: 2})
    torch.cuda.synchronize()
    assert rc == lib.EINVAL
    assert b"no-allocation limit" in L.cellato_last_error()
    assert int((a.buf != 0x5A).sum()) == 0 and int(b.buf.count_nonzero()) == 0


def test_noalloc_refuses_a_stream_under_capture(cuda):
    import torch
    from cellato_b200.device import DevicePlanes
    L = lib.load()
    a, b = DevicePlanes(1, 256, 64), DevicePlanes(1, 256, 64)
    x = torch.zeros(4, device="cuda")
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        x.add_(1)
        rc = _call([(0, 256, 64, 5, a.ptrs, b.ptrs)], stream=s.cuda_stream)
    assert rc == lib.EINVAL
    assert b"captured" in L.cellato_last_error()
    graph.replay()
    torch.cuda.synchronize()
    assert x.tolist() == [1.0] * 4
