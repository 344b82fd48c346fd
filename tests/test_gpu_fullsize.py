"""Properties at the workloads' full sizes, where the oracle is too slow to run:
the grids are seeded on the device, and kernels check one another.

* WireWorld and Greenberg-Hastings on 16384 x 16384 (the tiled W=64 workload):
  temporal runs with the depths, tile heights and row loops the autotuner picks
  agree with the single-step kernel.  The full-grid diff of the planes is zero
  and the checksums are equal.
* The same seeded grid run on the linear and on the tiled layout has the same
  checksum (the checksum is over cell values, not bytes).
* Cyclic and HPP fluid on 32768 x 32768 (the bit_planes workload): temporal
  k = 8 ... 32 at the default tile height (what the config-3 bench times) and
  the k = 1 temporal path agree with the single-step kernel.
The smaller sizes are pinned to the reference by the golden fixtures; these
tests pin the large ones to the small-size-verified kernels."""
import numpy as np
import pytest

from cellato_b200 import inputs, lib

pytestmark = pytest.mark.gpu


def seeded(rule, layout, X, Y, seed):
    from cellato_b200.device import DevicePlanes
    nb = inputs.PLANES[rule]
    a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
    lib.fill_random(layout, 64, nb, a.ptrs, X, Y, seed,
                    inputs.thresholds(inputs.REFERENCE_DENSITY[inputs.RULES[rule]]))
    return a, b


def run(rule, layout, X, Y, steps, seed, mode, k=1, tile_rows=0, loop=0, width=0, simple_kernel=0):
    a, b = seeded(rule, layout, X, Y, seed)
    if mode == "simple":
        in_b = lib.run_simple(rule, layout, 64, a.ptrs, b.ptrs, X, Y, 0, steps, simple_kernel=simple_kernel)
    else:
        in_b = lib.run_temporal(rule, layout, 64, a.ptrs, b.ptrs, X, Y, 0, steps, k, tile_rows, row_loop=loop,
                                words_per_lane=width)
    res = b if in_b else a
    other = a if in_b else b
    del other
    return res


def diff(nb, p, q):
    import torch
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    lib.diff_cells(nb, p.ptrs, q.ptrs, p.plane_bytes, out.data_ptr())
    torch.cuda.synchronize()
    return int(out.item())


def checksum(rule, layout, p, X, Y):
    import torch
    sums = torch.zeros(16, dtype=torch.int64, device="cuda")
    lib.checksum(rule, layout, 64, p.ptrs, X, Y, sums.data_ptr())
    torch.cuda.synchronize()
    return sums.cpu().tolist()


@pytest.mark.parametrize("rule,k,th,loop,width", [("wire", 8, 128, 1, 0), ("wire", 16, 0, 2, 0),
                                                  ("excitable", 16, 0, 2, 0), ("excitable", 8, 128, 1, 0),
                                                  ("excitable", 16, 192, 2, 2), ("wire", 16, 192, 1, 1),
                                                  ("wire", 12, 0, 3, 0), ("excitable", 16, 0, 3, 0),
                                                  ("excitable", 24, 256, 3, 2)])
def test_config2_size_temporal_equals_single_step(cuda, rule, k, th, loop, width):
    import torch
    r = lib.rule_id(rule)
    S, steps = 16384, 48
    ref = run(r, 1, S, S, steps, 42, "simple")
    got = run(r, 1, S, S, steps, 42, "temporal", k, th, loop, width)
    assert diff(inputs.PLANES[r], ref, got) == 0
    assert checksum(r, 1, ref, S, S) == checksum(r, 1, got, S, S)
    del ref, got
    torch.cuda.empty_cache()


def test_config2_size_layouts_agree_on_checksums(cuda):
    import torch
    S, steps = 16384, 40
    for rule in ("wire", "excitable"):
        r = lib.rule_id(rule)
        lin = run(r, 0, S, S, steps, 7, "temporal", 8)
        til = run(r, 1, S, S, steps, 7, "temporal", 8)
        c = checksum(r, 0, lin, S, S)
        assert c == checksum(r, 1, til, S, S), rule
        assert sum(c) > 0
        del lin, til
        torch.cuda.empty_cache()


@pytest.mark.parametrize("rule", ["cyclic", "fluid"])
def test_config3_size_temporal_equals_single_step(cuda, rule):
    """Every depth the config-3 workload lets the autotuner choose (k <= 32) at
    the library's default tile height and the three row loops, plus the k = 1
    single-step candidate, against the single-step kernel on 32768^2."""
    import torch
    r = lib.rule_id(rule)
    S, steps = 32768, 64
    ref = run(r, 0, S, S, steps, 42, "simple")
    for k, th, loop in ((16, 0, 2), (16, 0, 1), (24, 0, 2), (32, 0, 2), (12, 0, 2), (8, 0, 2), (1, 128, 1),
                        (16, 0, 3), (24, 0, 3), (8, 160, 3)):
        got = run(r, 0, S, S, steps, 42, "temporal", k, th, loop)
        assert diff(inputs.PLANES[r], ref, got) == 0, (rule, k, th, loop)
        del got
        torch.cuda.empty_cache()
    del ref
    torch.cuda.empty_cache()


@pytest.mark.parametrize("rule,layout,S,W", [("wire", 1, 16384, 32), ("excitable", 1, 16384, 64),
                                             ("cyclic", 0, 32768, 64), ("fluid", 0, 32768, 64),
                                             ("game-of-life", 0, 32768, 64), ("wire", 0, 32768, 64)])
def test_tma_single_step_equals_register_kernel(cuda, rule, layout, S, W):
    """The TMA-fed single-step kernel, at its default and every words-per-lane
    width the rule allows, against the register-band kernel at the workloads'
    full sizes, both word sizes of the tiled layout."""
    import torch
    from cellato_b200.device import DevicePlanes
    r = lib.rule_id(rule)
    nb = inputs.PLANES[r]
    steps = 7

    def run_kernel(kernel, width):
        a, b = DevicePlanes(nb, S, S), DevicePlanes(nb, S, S)
        lib.fill_random(layout, W, nb, a.ptrs, S, S, 9, inputs.thresholds(inputs.REFERENCE_DENSITY[rule]))
        in_b = lib.run_simple(r, layout, W, a.ptrs, b.ptrs, S, S, 0, steps, simple_kernel=kernel,
                              words_per_lane=width)
        return b if in_b else a

    ref = run_kernel(1, 0)
    for width in (0, 1, 2, 4):
        if (width == 2 and nb > 3) or (width == 4 and nb > 1):
            continue
        got = run_kernel(3, width)
        assert diff(nb, ref, got) == 0, width
        del got
        torch.cuda.empty_cache()
    assert lib.device_wait_timeouts() == 0
    del ref
    torch.cuda.empty_cache()
