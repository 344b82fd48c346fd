"""cellato_batch_run_noalloc -- the batched run for callers that must not
allocate device memory (an application that owns all device memory through its
own pool, a latency-critical loop that cannot take cudaMalloc's implicit
synchronisation, a fixed device-memory budget).  Its work list lives in a fixed
array of the library's device memory instead of a cudaMalloc'd buffer.

Checked through the C ABI against the existing batched entry point
(cellato_batch_create + cellato_batch_launch) on two calls in a row, with
different batches, so that the second call runs over the array the first one
left behind.  The path is integer bitwise work: results must be identical
(tolerance: exact).  This file is collected last on purpose."""
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
    for call, seed in enumerate((101, 202)):
        specs = batch_specs(seed, 20 + 9 * call)
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


def test_noalloc_rejects_batches_beyond_its_limit(cuda):
    import ctypes
    L = lib.load()
    n = 1025  # CELLATO_NOALLOC_MAX_GRIDS + 1
    arr = (lib.BatchGrid * n)()
    flags = (ctypes.c_int * n)()
    rc = L.cellato_batch_run_noalloc(0, 64, arr, n, None, None, flags)
    assert rc == lib.EINVAL
    assert b"no-allocation limit" in L.cellato_last_error()
