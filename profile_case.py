"""Run one hot-path configuration a fixed number of times, for profilers
(the command the ncu summaries under profiles/ were made with).

    python profile_case.py --rule excitable --layout tiled_bit_planes \
        --word-bits 64 --size 16384 --mode temporal --k 16 --launches 3

Inputs are the seeded workload grid of the rule, packed on the device.  Each
"launch" is one kernel launch: one step for --mode simple, k fused steps for
--mode temporal.  Prints the average launch time (CUDA events) and GCUPS.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "2026-cellato-smpt-journal_b200"))
from cellato_b200 import inputs, lib  # noqa: E402
from cellato_b200.device import DevicePlanes  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rule", default="excitable")
    ap.add_argument("--layout", default="tiled_bit_planes", choices=list(lib.LAYOUTS))
    ap.add_argument("--word-bits", type=int, default=64)
    ap.add_argument("--size", type=int, default=16384)
    ap.add_argument("--mode", default="temporal", choices=["simple", "temporal", "ops", "lop3", "batch"],
                    help="ops: the whole-grid operations (checksum, diff, random fill, packing, bit_array "
                         "conversion), each run --launches times; lop3: the ALU-pipe rate kernel "
                         "(lop3_rate.cu: one warm-up and three timed launches)")
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--tile-rows", type=int, default=0)
    ap.add_argument("--loop", type=int, default=0, help="temporal row loop (cellato_tune.row_loop)")
    ap.add_argument("--width", type=int, default=0, help="words per lane (cellato_tune.words_per_lane)")
    ap.add_argument("--simple-kernel", type=int, default=0, help="single-step kernel (cellato_tune.simple_kernel)")
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--grids", type=int, default=512, help="batch: grids in the batch (the batched workload's "
                                                            "distribution: sides 64-4096, aspect 1-4, 10 automata)")
    ap.add_argument("--max-steps", type=int, default=1000, help="batch: steps per grid uniform in 10..this")
    ap.add_argument("--warmup", type=int, default=1)
    a = ap.parse_args()

    r = lib.rule_id(a.rule)
    if a.mode == "lop3":
        from bench import lop3_rate
        print(json.dumps({"lop3_lane_ops_per_s": lop3_rate()}))
        return
    if a.mode == "ops":
        return ops(a, r)
    if a.mode == "batch":
        return batch(a)
    nb = lib.rule_planes(r)
    layout = lib.LAYOUTS[a.layout]
    X = Y = a.size
    cells = torch.from_numpy(inputs.workload_grid(inputs.RULES[r], X, Y, 42)).cuda()
    pa, pb = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
    pa.pack_from(cells, layout, a.word_bits)
    k = a.k if a.mode == "temporal" else 1

    def launch(n):
        if a.mode == "simple":
            return lib.run_simple(r, layout, a.word_bits, pa.ptrs, pb.ptrs, X, Y, 0, n, simple_kernel=a.simple_kernel,
                                  words_per_lane=a.width)
        return lib.run_temporal(r, layout, a.word_bits, pa.ptrs, pb.ptrs, X, Y, 0, n * k, k, a.tile_rows,
                                row_loop=a.loop, words_per_lane=a.width)

    launch(a.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    launch(a.launches)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.launches
    print(json.dumps({"rule": inputs.RULES[r], "layout": a.layout, "word_bits": a.word_bits, "size": a.size,
                      "mode": a.mode, "k": k, "ms_per_launch": round(ms, 4),
                      "gcups": round(X * Y * k / (ms * 1e-3) / 1e9, 1),
                      "algorithmic_bytes_per_launch": 2 * nb * X * Y // 8}))


def ops(a, r) -> None:
    """Each whole-grid operation --launches times after one warm-up, with its
    CUDA-event time and algorithmic bytes (what it must read and write)."""
    nb = lib.rule_planes(r)
    layout = lib.LAYOUTS[a.layout]
    X = Y = a.size
    pb = X * Y // 8
    p, q = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
    th = inputs.thresholds(inputs.REFERENCE_DENSITY[inputs.RULES[r]])
    cells = torch.empty((Y, X), dtype=torch.uint8, device="cuda")
    sums = torch.zeros(16, dtype=torch.int64, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    aw = 64
    arr = torch.empty(lib.load().cellato_bit_array_bytes(nb, aw, X, Y), dtype=torch.uint8, device="cuda")
    jobs = {
        "fill_random": (lambda: lib.fill_random(layout, a.word_bits, nb, p.ptrs, X, Y, 7, th), nb * pb),
        "checksum": (lambda: lib.checksum(r, layout, a.word_bits, p.ptrs, X, Y, sums.data_ptr()), nb * pb),
        "diff_cells": (lambda: lib.diff_cells(nb, p.ptrs, q.ptrs, pb, count.data_ptr()), 2 * nb * pb),
        "unpack_cells": (lambda: lib.unpack_cells(layout, a.word_bits, nb, p.ptrs, X, Y, cells.data_ptr()),
                         nb * pb + X * Y),
        "pack_cells": (lambda: lib.pack_cells(layout, a.word_bits, nb, cells.data_ptr(), X, Y, q.ptrs),
                       nb * pb + X * Y),
        "planes_to_bit_array": (lambda: lib.planes_to_bit_array(nb, layout, a.word_bits, p.ptrs, X, Y, aw,
                                                                arr.data_ptr()), nb * pb + arr.numel()),
        "bit_array_to_planes": (lambda: lib.bit_array_to_planes(nb, aw, arr.data_ptr(), X, Y, layout, a.word_bits,
                                                                q.ptrs), nb * pb + arr.numel()),
    }
    if X % (aw // nb):  # the bit_array layout needs whole words per row
        jobs.pop("planes_to_bit_array")
        jobs.pop("bit_array_to_planes")
    out = {}
    for name, (fn, byt) in jobs.items():
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.launches):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.launches
        out[name] = {"ms": round(ms, 4), "algorithmic_bytes": byt, "gbs": round(byt / (ms * 1e-3) / 1e9, 1)}
    print(json.dumps({"rule": inputs.RULES[r], "layout": a.layout, "word_bits": a.word_bits, "size": a.size,
                      "ops": out}))


def batch(a) -> None:
    """One batch of the batched workload's distribution (device-seeded, the same
    k for every rule), launched --launches times after --warmup launches."""
    import numpy as np
    from cellato_b200.batch import Batch
    rng = np.random.default_rng(42)
    layout, W = lib.LAYOUTS[a.layout], a.word_bits
    lo, hi = np.log(64), np.log(4096)
    grids, keep, cells = [], [], 0
    for i in range(a.grids):
        rule = int(rng.integers(0, 10))
        side = float(np.exp(rng.uniform(lo, hi)))
        aspect = float(rng.uniform(1.0, 4.0))
        X, Y = side * np.sqrt(aspect), side / np.sqrt(aspect)
        if rng.integers(0, 2):
            X, Y = Y, X
        X, Y = max(64, int(round(X / 64)) * 64), max(16, int(round(Y / 16)) * 16)
        steps = int(rng.integers(min(10, a.max_steps), a.max_steps + 1))
        nb = lib.rule_planes(rule)
        pa, pb = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
        lib.fill_random(layout, W, nb, pa.ptrs, X, Y, 1000 + i,
                        inputs.thresholds(inputs.REFERENCE_DENSITY[inputs.RULES[rule]]))
        grids.append((rule, X, Y, steps, pa.ptrs, pb.ptrs))
        keep.append((pa, pb))
        cells += X * Y * steps
    b = Batch(layout, W, grids, {r: a.k for r in range(10)})
    for _ in range(a.warmup):
        b.launch()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.launches):
        b.launch()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.launches
    print(json.dumps({"mode": "batch", "grids": a.grids, "k": a.k, "word_bits": W, "ms_per_launch": round(ms, 3),
                      "gcups": round(cells / (ms * 1e-3) / 1e9, 1), **b.info()}))


if __name__ == "__main__":
    main()
