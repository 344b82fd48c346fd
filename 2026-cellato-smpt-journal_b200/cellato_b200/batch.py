"""Batches of independent grids advanced by one CUDA-graph launch
(C ABI cellato_batch_*).

    b = Batch(layout, word_bits, [(rule, X, Y, steps, planes_a, planes_b), ...], k_per_rule)
    b.launch(stream)          # every grid advances its steps
    b.result_in_b(i)          # which buffer holds grid i's result
"""
from __future__ import annotations

import ctypes

from . import lib


class Batch:
    def __init__(self, layout: int, word_bits: int, grids, k_per_rule=None):
        L = lib.load()
        arr = (lib.BatchGrid * max(1, len(grids)))()
        for i, (rule, X, Y, steps, pa, pb) in enumerate(grids):
            arr[i].rule = lib.rule_id(rule)
            arr[i].x_cells, arr[i].y_cells, arr[i].steps = X, Y, steps
            for p, ptr in enumerate(pa):
                arr[i].planes_a[p] = ptr
            for p, ptr in enumerate(pb):
                arr[i].planes_b[p] = ptr
        ks, nk = lib.k_array(k_per_rule)
        h = ctypes.c_void_p()
        lib.check(L.cellato_batch_create(layout, word_bits, arr, len(grids), ks, nk, ctypes.byref(h)))
        self._h = h
        self.n = len(grids)

    def launch(self, stream: int = 0) -> None:
        lib.check(lib.load().cellato_batch_launch(self._h, stream))

    def result_in_b(self, i: int) -> int:
        v = ctypes.c_int()
        lib.check(lib.load().cellato_batch_result_in_b(self._h, i, ctypes.byref(v)))
        return v.value

    def info(self):
        n, w = ctypes.c_int(), ctypes.c_longlong()
        lib.check(lib.load().cellato_batch_info(self._h, ctypes.byref(n), ctypes.byref(w)))
        return {"kernel_launches": n.value, "work_items": w.value}

    def close(self) -> None:
        if self._h:
            lib.load().cellato_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_noalloc(layout: int, word_bits: int, grids, k_per_rule=None, stream: int = 0):
    """cellato_batch_run_noalloc: the batched run with its work list in the
    library's fixed device array (no device allocation).  grids as for Batch;
    returns the per-grid result_in_b flags."""
    L = lib.load()
    arr = (lib.BatchGrid * max(1, len(grids)))()
    for i, (rule, X, Y, steps, pa, pb) in enumerate(grids):
        arr[i].rule = lib.rule_id(rule)
        arr[i].x_cells, arr[i].y_cells, arr[i].steps = X, Y, steps
        for p, ptr in enumerate(pa):
            arr[i].planes_a[p] = ptr
        for p, ptr in enumerate(pb):
            arr[i].planes_b[p] = ptr
    ks, nk = lib.k_array(k_per_rule)
    flags = (ctypes.c_int * max(1, len(grids)))()
    lib.check(L.cellato_batch_run_noalloc(layout, word_bits, arr, len(grids), ks, nk, stream, flags))
    return [flags[i] for i in range(len(grids))]
