"""Run one hot-path configuration a fixed number of times, for profilers.

    python -m cellato_b200.profile_case --rule excitable --layout tiled_bit_planes \
        --word-bits 64 --size 16384 --mode temporal --k 16 --launches 3

Inputs are the seeded workload grid of the rule, packed on the device.  Each
"launch" is one kernel launch: one step for --mode simple, k fused steps for
--mode temporal.  Prints the average launch time (CUDA events) and GCUPS.
"""
from __future__ import annotations

import argparse
import json

import torch

from . import inputs, lib
from .device import DevicePlanes


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rule", default="excitable")
    ap.add_argument("--layout", default="tiled_bit_planes", choices=list(lib.LAYOUTS))
    ap.add_argument("--word-bits", type=int, default=64)
    ap.add_argument("--size", type=int, default=16384)
    ap.add_argument("--mode", default="temporal", choices=["simple", "temporal"])
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--tile-rows", type=int, default=0)
    ap.add_argument("--loop", type=int, default=0, help="temporal row loop (cellato_set_temporal_variant)")
    ap.add_argument("--width", type=int, default=0, help="temporal words per lane (cellato_set_temporal_width)")
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    a = ap.parse_args()

    r = lib.rule_id(a.rule)
    lib.set_temporal_variant(a.loop)
    lib.set_temporal_width(a.width)
    nb = lib.rule_planes(r)
    layout = lib.LAYOUTS[a.layout]
    X = Y = a.size
    cells = torch.from_numpy(inputs.workload_grid(inputs.RULES[r], X, Y, 42)).cuda()
    pa, pb = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
    pa.pack_from(cells, layout, a.word_bits)
    k = a.k if a.mode == "temporal" else 1

    def launch(n):
        if a.mode == "simple":
            return lib.run_simple(r, layout, a.word_bits, pa.ptrs, pb.ptrs, X, Y, 0, n)
        return lib.run_temporal(r, layout, a.word_bits, pa.ptrs, pb.ptrs, X, Y, 0, n * k, k, a.tile_rows)

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


if __name__ == "__main__":
    main()
