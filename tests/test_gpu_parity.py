"""GPU parity: the sm_100a kernels through the C ABI against the golden
fixtures (generated by the reference CPU standard path) and the oracle."""
import hashlib

import numpy as np
import pytest

from cellato_b200 import inputs, lib

from conftest import RULES

pytestmark = pytest.mark.gpu

# (layout, word_bits)
LAYOUTS = [(0, 32), (0, 64), (1, 32), (1, 64)]


def run_gpu(oracle, rule, layout, W, cells, steps, mode="simple", k=1, t0=0, tile_rows=0, row_loop=0,
            words_per_lane=0, simple_kernel=0):
    import torch
    from cellato_b200.device import DevicePlanes
    Y, X = cells.shape
    nb = inputs.PLANES[rule]
    a = DevicePlanes(nb, X, Y)
    b = DevicePlanes(nb, X, Y)
    a.upload(oracle.pack(layout, W, nb, cells))
    if mode == "simple":
        in_b = lib.run_simple(rule, layout, W, a.ptrs, b.ptrs, X, Y, t0, steps, simple_kernel=simple_kernel,
                              words_per_lane=words_per_lane)
    else:
        in_b = lib.run_temporal(rule, layout, W, a.ptrs, b.ptrs, X, Y, t0, steps, k, tile_rows,
                                row_loop=row_loop, words_per_lane=words_per_lane)
    torch.cuda.synchronize()
    res = (b if in_b else a).download()
    return oracle.unpack(layout, W, nb, res, X, Y)


@pytest.mark.parametrize("layout,W", LAYOUTS)
def test_simple_small_golden(cuda, oracle, golden_small, layout, W):
    for case, cin, cout in golden_small:
        r = RULES.index(case["rule"])
        out = run_gpu(oracle, r, layout, W, cin, case["steps"])
        assert np.array_equal(out, cout), (case["key"], case["rule"], int((out != cout).sum()))


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 8, 16, 24, 32])
@pytest.mark.parametrize("layout,W", LAYOUTS)
def test_temporal_small_golden(cuda, oracle, golden_small, layout, W, k):
    for case, cin, cout in golden_small:
        r = RULES.index(case["rule"])
        out = run_gpu(oracle, r, layout, W, cin, case["steps"], mode="temporal", k=k)
        assert np.array_equal(out, cout), (case["key"], case["rule"], k, int((out != cout).sum()))


@pytest.mark.parametrize("width", [1, 2])
@pytest.mark.parametrize("loop", [1, 2, 3])
@pytest.mark.parametrize("k", [2, 3, 8, 24, 32])
@pytest.mark.parametrize("layout,W", LAYOUTS)
def test_temporal_row_loops(cuda, oracle, golden_small, layout, W, k, loop, width):
    """The three row loops (cellato_tune.row_loop: row by row, hoisted, two
    steps per sweep -- odd k ends with a single step) and both tile widths
    (cellato_tune.words_per_lane) of the temporal kernel.  The tiles are the
    shortest allowed, so late steps leave warps bands of zero to four rows."""
    # the shortest tile that leaves 16 interior rows below the two k-row halos
    th = max(48, 2 * ((k + 7) // 8 * 8) + 16)
    for case, cin, cout in golden_small:
        r = RULES.index(case["rule"])
        out = run_gpu(oracle, r, layout, W, cin, case["steps"], mode="temporal", k=k, tile_rows=th, row_loop=loop,
                      words_per_lane=width)
        assert np.array_equal(out, cout), (case["key"], case["rule"], k, loop, width)


@pytest.mark.parametrize("mode,k,loop", [("simple", 1, 0), ("temporal", 3, 0), ("temporal", 8, 0), ("temporal", 3, 3),
                                         ("temporal", 8, 3)])
@pytest.mark.parametrize("t0", [1, 2, 7])
def test_step_parity_offsets(cuda, oracle, mode, k, loop, t0):
    """alternate_algorithms and Margolus phase follow the global step number
    (also when two steps share a sweep, loop 3)."""
    rng = np.random.default_rng(t0)
    for r in range(10):
        cells = rng.integers(0, inputs.STATES[r], size=(40, 128), dtype=np.uint8)
        want = oracle.run(r, cells, 11, t0=t0)
        for layout, W in [(0, 32), (1, 64)]:
            if layout == 1 and 40 % (W // 8):
                continue
            got = run_gpu(oracle, r, layout, W, cells, 11, mode=mode, k=k, t0=t0, row_loop=loop)
            assert np.array_equal(got, want), (RULES[r], layout, W, t0, loop)


def test_odd_heights_and_narrow_rows(cuda, oracle):
    """Ragged shapes: odd Y (linear), one-word rows, rows narrower than a warp."""
    rng = np.random.default_rng(11)
    for r in range(10):
        for X, Y in [(32, 1), (32, 3), (64, 7), (96, 5), (160, 33), (4096, 9)]:
            cells = rng.integers(0, inputs.STATES[r], size=(Y, X), dtype=np.uint8)
            want = oracle.run(r, cells, 6)
            assert np.array_equal(run_gpu(oracle, r, 0, 32, cells, 6), want), (RULES[r], X, Y)
            assert np.array_equal(run_gpu(oracle, r, 0, 32, cells, 6, mode="temporal", k=4), want), (RULES[r], X, Y)


def test_large_golden(cuda, oracle, golden_large):
    """Workload-sized crops, full-grid SHA-256 against the reference's output."""
    plans = {
        "game-of-life": [(0, 64, "simple", 1), (0, 64, "temporal", 8), (1, 64, "temporal", 8)],
        "wire": [(1, 64, "temporal", 8), (1, 64, "simple", 1), (1, 32, "temporal", 5)],
        "excitable": [(1, 64, "temporal", 8), (1, 32, "simple", 1)],
        "cyclic": [(0, 64, "simple", 1), (0, 32, "temporal", 4)],
        "fluid": [(0, 64, "simple", 1), (0, 64, "temporal", 7), (1, 64, "temporal", 8)],
    }
    for case in golden_large:
        rule = case["rule"]
        r = RULES.index(rule)
        if case["generator"] == "workload":
            cells = inputs.workload_grid(rule, case["X"], case["Y"], case["seed"])
        else:
            cells = inputs.reference_density_grid(rule, case["X"], case["Y"], case["seed"])
        for layout, W, mode, k in plans.get(rule, [(0, 64, "simple", 1), (1, 64, "temporal", 6)]):
            out = run_gpu(oracle, r, layout, W, cells, case["steps"], mode=mode, k=k)
            assert hashlib.sha256(out.tobytes()).hexdigest() == case["sha256_out"], (rule, layout, W, mode, k)


def test_temporal_tile_too_large(cuda):
    a = [0x1000]
    b = [0x2000]
    with pytest.raises(lib.CellatoError) as e:
        lib.run_temporal("game-of-life", 0, 64, a, b, 64, 8, 0, 4, k=4, tile_rows=8 * 1000)
    assert e.value.status == lib.ESMEM


@pytest.mark.parametrize("layout,W", LAYOUTS)
def test_device_pack_matches_reference_layout(cuda, oracle, layout, W):
    """cellato_pack_cells writes the reference's plane bytes; unpack inverts it."""
    import torch
    from cellato_b200.device import DevicePlanes
    rng = np.random.default_rng(W + layout)
    for nb in (1, 2, 3, 4, 5):
        for X, Y in [(64, 8), (192, 24), (1024, 64)]:
            cells = rng.integers(0, 1 << nb, size=(Y, X), dtype=np.uint8)
            d = DevicePlanes(nb, X, Y)
            d.pack_from(torch.from_numpy(cells).cuda(), layout, W)
            torch.cuda.synchronize()
            assert np.array_equal(d.download(), oracle.pack(layout, W, nb, cells)), (nb, X, Y)
            assert np.array_equal(d.unpack(layout, W).cpu().numpy(), cells), (nb, X, Y)


def test_streaming_kernel_shapes_and_no_wait_timeouts(cuda, oracle):
    """The bulk-copy streaming kernel (linear rows of 16-byte multiples):
    segments shorter than a warp, partial last segments, wrapped halos, tall
    and one-row grids; afterwards no bounded device wait may have given up."""
    rng = np.random.default_rng(21)
    for r in range(10):
        for X, Y in [(128, 1), (128, 5), (256, 17), (384, 9), (4096 + 128, 13), (8192, 33)]:
            cells = rng.integers(0, inputs.STATES[r], size=(Y, X), dtype=np.uint8)
            want = oracle.run(r, cells, 5, t0=3)
            for W in (32, 64):
                got = run_gpu(oracle, r, 0, W, cells, 5, t0=3, simple_kernel=2)
                assert np.array_equal(got, want), (RULES[r], X, Y, W)
    assert lib.device_wait_timeouts() == 0


@pytest.mark.parametrize("layout,W", LAYOUTS)
@pytest.mark.parametrize("width", [0, 1, 2, 4])
def test_tma_single_step_kernel(cuda, oracle, layout, W, width):
    """The TMA-fed single-step kernel (cellato_tune.simple_kernel = 3) at its
    default and every words-per-lane width a rule allows (strips of 4096 cells
    at one word per lane, 8192 at two or four; narrower rows fall back to the
    register kernel): every rule, one and two strips per row, heights from one
    stage to several CTAs per strip, wrapped halos, odd step offsets."""
    rng = np.random.default_rng(31 + layout + W + width)
    for r in range(10):
        nb = inputs.PLANES[r]
        if (width == 2 and nb > 3) or (width == 4 and nb > 1):
            continue
        for X, Y in [(4096, 96), (8192, 40), (4096, 264), (16384, 24), (8192, 136)]:
            cells = rng.integers(0, inputs.STATES[r], size=(Y, X), dtype=np.uint8)
            want = oracle.run(r, cells, 5, t0=3)
            got = run_gpu(oracle, r, layout, W, cells, 5, t0=3, simple_kernel=3, words_per_lane=width)
            assert np.array_equal(got, want), (RULES[r], X, Y, layout, W, width)
    assert lib.device_wait_timeouts() == 0
