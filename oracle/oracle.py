"""Test infrastructure only: ctypes access to the oracle.

* ``Oracle``    -- the plain-C restatement (oracle/cellato_oracle.c, liboracle.so).
* ``RefOracle`` -- the reference's own CPU code compiled by oracle/Makefile into
  oracle/_ref/libcellato_ref.so (present where the reference tree was available
  at build time; it travels with the repository snapshot).
* ``RefCustomOracle`` -- the reference's standard path instantiated for the
  custom rules of tests/cpp/custom_rules.hpp (oracle/_ref/libcellato_ref_custom.so).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this
module, and only as the checker or the timed CPU baseline.  Cells are uint8
dictionary indices (the integer the bit planes encode).
"""
from __future__ import annotations

import ctypes
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libcellato_ref.so")
REF_CUSTOM_PATH = os.path.join(HERE, "_ref", "libcellato_ref_custom.so")

RULES = ["game-of-life", "forest-fire", "wire", "excitable", "brian",
         "maze", "cyclic", "fluid", "critters", "traffic"]

_u8p = ctypes.POINTER(ctypes.c_uint8)


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u8p)


class Oracle:
    """The C restatement of the reference standard CPU path."""

    def __init__(self, path: str = LIB_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        lib = ctypes.CDLL(path)
        lib.oracle_run.argtypes = [ctypes.c_int, _u8p, _u8p, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.oracle_pack.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _u8p,
                                    ctypes.c_int, ctypes.c_int, _u8p]
        lib.oracle_unpack.argtypes = lib.oracle_pack.argtypes
        lib.oracle_checksum.argtypes = [ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_uint64)]
        lib.oracle_rule_name.restype = ctypes.c_char_p
        lib.oracle_rule_from_name.argtypes = [ctypes.c_char_p]
        self.lib = lib

    def planes(self, rule: int) -> int:
        return self.lib.oracle_planes(rule)

    def states(self, rule: int) -> int:
        return self.lib.oracle_states(rule)

    def state_value(self, rule: int, index: int) -> int:
        return self.lib.oracle_state_value(rule, index)

    def run(self, rule: int, cells: np.ndarray, steps: int, t0: int = 0, threads: int = 0) -> np.ndarray:
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        out = np.empty_like(cells)
        threads = threads or (os.cpu_count() or 1)
        rc = self.lib.oracle_run(rule, _ptr(cells), _ptr(out), X, Y, t0, steps, threads)
        if rc != 0:
            raise RuntimeError(f"oracle_run failed: {rc}")
        return out

    def pack(self, layout: int, word_bits: int, nb: int, cells: np.ndarray) -> np.ndarray:
        """Returns an array of shape (nb, X*Y/8) uint8: the planes as bytes."""
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        out = np.zeros((nb, X * Y // 8), dtype=np.uint8)
        rc = self.lib.oracle_pack(layout, word_bits, nb, _ptr(cells), X, Y, _ptr(out))
        if rc != 0:
            raise ValueError(f"oracle_pack rejected layout={layout} W={word_bits} X={X} Y={Y}")
        return out

    def unpack(self, layout: int, word_bits: int, nb: int, planes: np.ndarray, X: int, Y: int) -> np.ndarray:
        planes = np.ascontiguousarray(planes, dtype=np.uint8)
        out = np.empty((Y, X), dtype=np.uint8)
        rc = self.lib.oracle_unpack(layout, word_bits, nb, _ptr(planes), X, Y, _ptr(out))
        if rc != 0:
            raise ValueError("oracle_unpack rejected its arguments")
        return out

    @staticmethod
    def pack_bit_array(nb: int, word_bits: int, cells: np.ndarray) -> np.ndarray:
        """The reference's bit_array layout (include/memory/bit_array_grid.hpp:
        298-310 set_cell_at_index, :143-159): cells in row-major order,
        cells_per_word = word_bits // nb, cell i in word i // cpw at bit
        (i % cpw) * nb; the word count rounds up.  Returns the words."""
        cpw = word_bits // nb
        flat = np.ascontiguousarray(cells, dtype=np.uint8).reshape(-1).astype(np.uint64)
        words = (flat.size + cpw - 1) // cpw
        pad = np.zeros(words * cpw, dtype=np.uint64)
        pad[:flat.size] = flat
        shifts = np.arange(cpw, dtype=np.uint64) * np.uint64(nb)
        w = np.bitwise_or.reduce(pad.reshape(words, cpw) << shifts, axis=1)
        return w.astype(np.uint32 if word_bits == 32 else np.uint64)

    @staticmethod
    def unpack_bit_array(nb: int, word_bits: int, words: np.ndarray, X: int, Y: int) -> np.ndarray:
        """Inverse of pack_bit_array (get_cell_at_index, bit_array_grid.hpp:312-320)."""
        cpw = word_bits // nb
        w = np.asarray(words).astype(np.uint64)
        shifts = np.arange(cpw, dtype=np.uint64) * np.uint64(nb)
        cells = (w[:, None] >> shifts) & np.uint64((1 << nb) - 1)
        return cells.reshape(-1)[:X * Y].astype(np.uint8).reshape(Y, X)

    def checksum(self, rule: int, cells: np.ndarray) -> str:
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        out = (ctypes.c_uint64 * 16)()
        self.lib.oracle_checksum(rule, _ptr(cells), X, Y, out)
        return "-".join(str(v) for v in out)


class RefOracle:
    """The reference's own CPU code (compiled from the reference tree)."""

    def __init__(self, path: str = REF_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        lib = ctypes.CDLL(path)
        lib.cref_run_standard.argtypes = [ctypes.c_int, _u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.cref_run_standard_mt.argtypes = [ctypes.c_int, _u8p, _u8p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int]
        lib.cref_run_bit_planes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _u8p, _u8p,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.cref_pack.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _u8p, ctypes.c_int,
                                  ctypes.c_int, _u8p]
        lib.cref_pack.restype = ctypes.c_longlong
        lib.cref_pack_bit_array.argtypes = [ctypes.c_int, ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int, _u8p]
        lib.cref_pack_bit_array.restype = ctypes.c_longlong
        lib.cref_reference_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _u8p]
        lib.cref_checksum.argtypes = [ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                      ctypes.c_int]
        lib.cref_rule_name.restype = ctypes.c_char_p
        self.lib = lib

    def name(self, rule: int) -> str:
        return self.lib.cref_rule_name(rule).decode()

    def planes(self, rule: int) -> int:
        return self.lib.cref_needed_bits(rule)

    def states(self, rule: int) -> int:
        return self.lib.cref_number_of_states(rule)

    def state_value(self, rule: int, index: int) -> int:
        return self.lib.cref_state_value(rule, index)

    def run_standard(self, rule: int, cells: np.ndarray, steps: int, threads: int = 1) -> np.ndarray:
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        out = np.empty_like(cells)
        if threads == 1:
            rc = self.lib.cref_run_standard(rule, _ptr(cells), _ptr(out), X, Y, steps)
        else:
            rc = self.lib.cref_run_standard_mt(rule, _ptr(cells), _ptr(out), X, Y, steps, threads)
        if rc != 0:
            raise RuntimeError(f"reference standard run failed: {rc}")
        return out

    def run_bit_planes(self, rule: int, word_bits: int, tiled: bool, cells: np.ndarray, steps: int) -> np.ndarray:
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        out = np.empty_like(cells)
        rc = self.lib.cref_run_bit_planes(rule, word_bits, int(tiled), _ptr(cells), _ptr(out), X, Y, steps)
        if rc != 0:
            raise RuntimeError(f"reference bit-plane run failed: {rc}")
        return out

    def pack(self, rule: int, word_bits: int, tiled: bool, cells: np.ndarray) -> np.ndarray:
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        nb = self.planes(rule)
        out = np.zeros((nb, X * Y // 8), dtype=np.uint8)
        r = self.lib.cref_pack(rule, word_bits, int(tiled), _ptr(cells), X, Y, _ptr(out))
        if r < 0:
            raise RuntimeError("reference pack failed")
        return out

    def pack_bit_array(self, rule: int, word_bits: int, cells: np.ndarray) -> np.ndarray:
        """Words of the reference's own bit_array grid built from `cells`."""
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        nb = self.planes(rule)
        cpw = word_bits // nb
        words = (X * Y + cpw - 1) // cpw
        out = np.zeros(words, dtype=np.uint32 if word_bits == 32 else np.uint64)
        r = self.lib.cref_pack_bit_array(rule, word_bits, _ptr(cells), X, Y, out.ctypes.data_as(_u8p))
        if r < 0:
            raise RuntimeError("reference bit_array pack failed")
        return out

    def reference_init(self, rule: int, X: int, Y: int, seed: int) -> np.ndarray:
        out = np.empty((Y, X), dtype=np.uint8)
        rc = self.lib.cref_reference_init(rule, X, Y, seed, _ptr(out))
        if rc != 0:
            raise RuntimeError("reference init failed")
        return out

    def checksum(self, rule: int, cells: np.ndarray) -> str:
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        buf = ctypes.create_string_buffer(1024)
        n = self.lib.cref_checksum(rule, _ptr(cells), X, Y, buf, 1024)
        if n < 0:
            raise RuntimeError("reference checksum failed")
        return buf.value.decode()


class RefCustomOracle:
    """The reference's CPU standard path on the custom rules (rules outside both
    the reference and the B200 library, tests/cpp/custom_rules.hpp)."""

    def __init__(self, path: str = REF_CUSTOM_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        lib = ctypes.CDLL(path)
        lib.cref_custom_name.restype = ctypes.c_char_p
        lib.cref_custom_run.argtypes = [ctypes.c_int, _u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        self.lib = lib

    def count(self) -> int:
        return self.lib.cref_custom_count()

    def name(self, which: int) -> str:
        return self.lib.cref_custom_name(which).decode()

    def states(self, which: int) -> int:
        return self.lib.cref_custom_states(which)

    def run_standard(self, which: int, cells: np.ndarray, steps: int) -> np.ndarray:
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        Y, X = cells.shape
        out = np.empty_like(cells)
        if self.lib.cref_custom_run(which, _ptr(cells), _ptr(out), X, Y, steps) != 0:
            raise RuntimeError("reference standard run of a custom rule failed")
        return out
