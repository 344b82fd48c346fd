"""Batched execution (cellato_batch_*): many grids of mixed rules, sizes and
step counts in one CUDA-graph launch, each bit-exact against the oracle and
against a plain per-grid temporal run."""
import numpy as np
import pytest

from cellato_b200 import inputs, lib

from conftest import RULES

pytestmark = pytest.mark.gpu


def make_grids(rng, n, layout, W, max_side=320):
    out = []
    for i in range(n):
        r = int(rng.integers(0, 10))
        X = int(rng.integers(1, max_side // 64 + 1)) * 64
        Y = int(rng.integers(1, max_side // 8 + 1)) * 8
        steps = int(rng.integers(0, 40))
        cells = rng.integers(0, inputs.STATES[r], size=(Y, X), dtype=np.uint8)
        out.append((r, X, Y, steps, cells))
    return out


@pytest.mark.parametrize("layout,W", [(1, 64), (0, 32)])
def test_batch_matches_oracle_and_single_runs(cuda, oracle, layout, W):
    import torch
    from cellato_b200.batch import Batch
    from cellato_b200.device import DevicePlanes
    rng = np.random.default_rng(5 + layout)
    specs = make_grids(rng, 48, layout, W)
    bufs = []
    for r, X, Y, steps, cells in specs:
        nb = inputs.PLANES[r]
        a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
        a.upload(oracle.pack(layout, W, nb, cells))
        bufs.append((a, b))
    ks = {r: [3, 4, 5, 6, 7, 8, 2, 4, 5, 3][r] for r in range(10)}
    batch = Batch(layout, W, [(r, X, Y, s, a.ptrs, b.ptrs) for (r, X, Y, s, _), (a, b) in zip(specs, bufs)], ks)
    batch.launch()
    torch.cuda.synchronize()
    for i, ((r, X, Y, steps, cells), (a, b)) in enumerate(zip(specs, bufs)):
        res = (b if batch.result_in_b(i) else a).download()
        got = oracle.unpack(layout, W, inputs.PLANES[r], res, X, Y)
        assert np.array_equal(got, oracle.run(r, cells, steps)), (i, RULES[r], X, Y, steps)
        # the same grid alone through the single-grid temporal traverser
        nb = inputs.PLANES[r]
        c, d = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
        c.upload(oracle.pack(layout, W, nb, cells))
        in_d = lib.run_temporal(r, layout, W, c.ptrs, d.ptrs, X, Y, 0, steps, ks[r])
        torch.cuda.synchronize()
        assert np.array_equal((d if in_d else c).download(), res), i
    info = batch.info()
    assert info["kernel_launches"] >= 1 and info["work_items"] >= len(specs) - sum(1 for s in specs if s[3] == 0)
    # a second launch continues from the results (ping-pong alternates)
    batch.close()


def test_batch_rejects_bad_grids(cuda):
    from cellato_b200.batch import Batch
    with pytest.raises(lib.CellatoError):
        Batch(0, 64, [(0, 96, 8, 5, [0x1000], [0x2000])])
    with pytest.raises(lib.CellatoError):
        Batch(0, 64, [(11, 64, 8, 5, [0x1000], [0x2000])])
