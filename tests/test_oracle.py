"""The oracle (C restatement of the reference CPU standard path) against the
golden fixtures generated from the reference itself."""
import hashlib

import numpy as np
import pytest

from cellato_b200 import inputs

from conftest import RULES


def test_rule_metadata(oracle):
    assert [oracle.planes(r) for r in range(10)] == inputs.PLANES
    assert [oracle.states(r) for r in range(10)] == inputs.STATES


def test_small_golden(oracle, golden_small):
    assert len(golden_small) == 70
    for case, cin, cout in golden_small:
        r = RULES.index(case["rule"])
        out = oracle.run(r, cin, case["steps"])
        assert np.array_equal(out, cout), case["key"]
        assert oracle.checksum(r, out) == case["checksum"], case["key"]


@pytest.mark.parametrize("rule", RULES)
def test_large_golden(oracle, golden_large, rule):
    for case in golden_large:
        if case["rule"] != rule:
            continue
        if case["generator"] == "workload":
            cells = inputs.workload_grid(rule, case["X"], case["Y"], case["seed"])
        else:
            cells = inputs.reference_density_grid(rule, case["X"], case["Y"], case["seed"])
        assert hashlib.sha256(cells.tobytes()).hexdigest() == case["sha256_in"], "input generator drifted"
        out = oracle.run(RULES.index(rule), cells, case["steps"])
        assert hashlib.sha256(out.tobytes()).hexdigest() == case["sha256_out"]
        assert oracle.checksum(RULES.index(rule), out) == case["checksum"]


@pytest.mark.parametrize("layout,W", [(0, 32), (0, 64), (1, 32), (1, 64)])
def test_pack_roundtrip(oracle, layout, W):
    rng = np.random.default_rng(5)
    for nb in (1, 2, 3, 5):
        cells = rng.integers(0, 1 << nb, size=(16, 128), dtype=np.uint8)
        planes = oracle.pack(layout, W, nb, cells)
        assert planes.shape == (nb, 16 * 128 // 8)
        assert np.array_equal(oracle.unpack(layout, W, nb, planes, 128, 16), cells)


def test_layout_known_answers(oracle):
    # linear: cell (x, y) -> plane bit (y * X + x), least significant bit leftmost
    cells = np.zeros((8, 64), dtype=np.uint8)
    cells[0, 0] = 1
    cells[1, 33] = 1
    p = oracle.pack(0, 32, 1, cells)[0].view(np.uint32)
    assert p[0] == 1 and p[3] == 2
    # tiled 8x8: tile (0,0) bit (y%8)*8 + x%8
    t = oracle.pack(1, 64, 1, cells)[0].view(np.uint64)
    assert t[0] == 1 and t[4] == (1 << (8 + 1))
    # tiled 8x4: cell (33, 1) -> tile (4, 0), bit 1*8 + 1
    t32 = oracle.pack(1, 32, 1, cells)[0].view(np.uint32)
    assert t32[4] == (1 << 9)


def test_bit_array_layout_matches_reference(oracle):
    """The oracle's restatement of the bit_array layout against the words of the
    reference's own bit_array grid, for every rule and both word sizes."""
    from oracle import RefOracle
    try:
        ref = RefOracle()
    except FileNotFoundError:
        pytest.skip("reference CPU library not built")
    rng = np.random.default_rng(17)
    for r in range(10):
        nb = oracle.planes(r)
        for W in (32, 64):
            cpw = W // nb
            X, Y = cpw * 7, 13
            cells = rng.integers(0, oracle.states(r), size=(Y, X), dtype=np.uint8)
            want = ref.pack_bit_array(r, W, cells)
            got = oracle.pack_bit_array(nb, W, cells)
            assert got.dtype == want.dtype and np.array_equal(got, want), (RULES[r], W)
            assert np.array_equal(oracle.unpack_bit_array(nb, W, got, X, Y), cells)
