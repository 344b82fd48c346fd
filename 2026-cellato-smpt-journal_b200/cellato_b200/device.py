"""Device-resident bit planes held in torch CUDA memory.

torch is used here only as the device allocator and stream provider; every
computation on the planes goes through the C ABI.
"""
from __future__ import annotations

import numpy as np
import torch

from . import lib

ALIGN = 256


def _round_up(n: int, a: int) -> int:
    return (n + a - 1) // a * a


class DevicePlanes:
    """nb planes of X*Y/8 bytes, each starting on a 256-byte boundary."""

    def __init__(self, nb: int, X: int, Y: int, device: str | torch.device = "cuda"):
        self.nb, self.X, self.Y = nb, X, Y
        self.plane_bytes = X * Y // 8
        self.stride = _round_up(max(self.plane_bytes, 16), ALIGN)
        self.buf = torch.zeros(nb * self.stride + ALIGN, dtype=torch.uint8, device=device)
        base = self.buf.data_ptr()
        self.offset = (-base) % ALIGN
        self.ptrs = [base + self.offset + p * self.stride for p in range(nb)]

    def view(self, p: int) -> torch.Tensor:
        o = self.offset + p * self.stride
        return self.buf[o:o + self.plane_bytes]

    def upload(self, planes: np.ndarray) -> None:
        """planes: (nb, X*Y/8) uint8 host array."""
        assert planes.shape == (self.nb, self.plane_bytes), planes.shape
        for p in range(self.nb):
            self.view(p).copy_(torch.from_numpy(np.ascontiguousarray(planes[p])))

    def download(self) -> np.ndarray:
        out = np.empty((self.nb, self.plane_bytes), dtype=np.uint8)
        for p in range(self.nb):
            out[p] = self.view(p).cpu().numpy()
        return out

    # ---- device packing (C ABI cellato_pack_cells / cellato_unpack_cells)
    def pack_from(self, cells: torch.Tensor, layout: int, word_bits: int, stream: int = 0) -> None:
        """cells: (Y, X) uint8 CUDA tensor of state indices."""
        assert cells.dtype == torch.uint8 and cells.is_cuda and cells.is_contiguous()
        assert tuple(cells.shape) == (self.Y, self.X)
        lib.pack_cells(layout, word_bits, self.nb, cells.data_ptr(), self.X, self.Y, self.ptrs, stream)

    def unpack(self, layout: int, word_bits: int, stream: int = 0) -> torch.Tensor:
        cells = torch.empty((self.Y, self.X), dtype=torch.uint8, device=self.buf.device)
        lib.unpack_cells(layout, word_bits, self.nb, self.ptrs, self.X, self.Y, cells.data_ptr(), stream)
        return cells
