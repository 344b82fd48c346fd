"""Device conversion between the reference's bit_array layout and bit planes
(cellato_bit_array_to_planes / cellato_planes_to_bit_array) against the
oracle's bit_array restatement, which tests/test_oracle.py pins to the words of
the reference's own bit_array grid: every rule, both bit_array word sizes, every
plane layout and word size, and widths whose words hold a number of cells
that is not a power of two."""
import numpy as np
import pytest

from cellato_b200 import inputs, lib

from conftest import RULES

pytestmark = pytest.mark.gpu

PLANE_FORMATS = [(0, 32), (0, 64), (1, 32), (1, 64)]


@pytest.mark.parametrize("aw", [32, 64])
@pytest.mark.parametrize("layout,W", PLANE_FORMATS)
def test_bit_array_conversions(cuda, oracle, aw, layout, W):
    import torch
    from cellato_b200.device import DevicePlanes
    rng = np.random.default_rng(aw + 3 * layout + W)
    for r in range(10):
        nb = inputs.PLANES[r]
        cpw = aw // nb
        X = int(np.lcm(np.lcm(cpw, 64), W))
        Y = 48
        cells = rng.integers(0, inputs.STATES[r], size=(Y, X), dtype=np.uint8)
        words = oracle.pack_bit_array(nb, aw, cells)
        assert lib.load().cellato_bit_array_bytes(nb, aw, X, Y) == words.nbytes
        dev_words = torch.from_numpy(words.view(np.uint8).copy()).cuda()
        p = DevicePlanes(nb, X, Y)
        lib.bit_array_to_planes(nb, aw, dev_words.data_ptr(), X, Y, layout, W, p.ptrs)
        torch.cuda.synchronize()
        assert np.array_equal(oracle.unpack(layout, W, nb, p.download(), X, Y), cells), (RULES[r], aw, layout, W)
        back = torch.full_like(dev_words, 0xA5)
        lib.planes_to_bit_array(nb, layout, W, p.ptrs, X, Y, aw, back.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(back.cpu().numpy(), words.view(np.uint8)), (RULES[r], aw, layout, W)


def test_bit_array_rejects_widths_that_split_a_word(cuda):
    import torch
    from cellato_b200.device import DevicePlanes
    buf = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    p = DevicePlanes(3, 64, 8)
    with pytest.raises(lib.CellatoError):
        lib.bit_array_to_planes(3, 32, buf.data_ptr(), 64, 8, 0, 32, p.ptrs)   # 64 % (32 // 3) != 0
