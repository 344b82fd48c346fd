"""Autotuner: picks the traverser configuration per automaton and grid size.

The reference leaves (temporal_steps, temporal_tile_size_y, cuda_block_size_y)
to the user and sweeps them with run_all.py (src/_scripts/cluster_run/
run_all.py:9-24).  Here the choice is measured on the device: each candidate --
the single-step kernel, or the temporal kernel with k fused steps -- runs a
short burst on the caller's own device planes and the fastest per cell-step
wins.  Results are cached per (rule, layout, word size, size class, device) in
memory and in a JSON file, so a server or batch launcher pays the search once.
"""
from __future__ import annotations

import json
import math
import os
import threading

from . import lib

# (mode, k[, tile_rows[, row loop]]); tile_rows 0 = the library's default height
# for k; row loop as cellato_tune.row_loop (0 = default)
# Single-step candidates: the two single-step kernels and the temporal kernel at
# k = 1 (one step per launch through a shared-memory tile), which for rules with
# many planes or long networks reaches more of the HBM roofline.
SINGLE_STEP_CANDIDATES = (("simple_register", 1), ("simple_stream", 1)) + tuple(
    ("temporal", 1, th, loop, width) for th in (0, 96, 128, 192) for loop in (1, 2) for width in (1, 2))
# (mode, k, tile_rows, row loop, words per lane); words per lane as
# cellato_tune.words_per_lane (1 or 2; two words per lane exist only for rules of
# up to three planes, and are skipped for the others)
DEFAULT_CANDIDATES = SINGLE_STEP_CANDIDATES + (("temporal", 2),) + tuple(
    ("temporal", k, th, loop, width) for k in (4, 6, 8, 12, 16, 24) for th in (0, 96, 128, 160, 192, 256, 320)
    for loop in (1, 2) for width in (1, 2))
_VARIANT = {"simple": 0, "simple_register": 1, "simple_stream": 2}

_lock = threading.Lock()
_memo: dict = {}


def size_class(X: int, Y: int) -> int:
    """log2 of the cell count, rounded: grids within a factor ~1.4 share a tuning."""
    return int(round(math.log2(max(1, X * Y))))


def cache_path() -> str:
    return os.environ.get("CELLATO_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "cellato_b200_autotune.json"))


def _key(rule: int, layout: int, word_bits: int, X: int, Y: int, device_name: str) -> str:
    return f"v8/{rule}/{layout}/{word_bits}/{size_class(X, Y)}/{device_name}"


def _load_file() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_file(key: str, value: dict) -> None:
    try:
        d = _load_file()
        d[key] = value
        os.makedirs(os.path.dirname(cache_path()), exist_ok=True)
        tmp = cache_path() + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1)
        os.replace(tmp, cache_path())
    except OSError:
        pass


def run(choice: dict, rule: int, layout: int, word_bits: int, planes_a, planes_b, X: int, Y: int, t0: int,
        steps: int, stream: int = 0) -> int:
    """Run `steps` steps with a tuned choice; returns 1 if the result is in planes_b."""
    if choice["mode"] in _VARIANT:
        return lib.run_simple(rule, layout, word_bits, planes_a, planes_b, X, Y, t0, steps, stream,
                              simple_kernel=_VARIANT[choice["mode"]])
    return lib.run_temporal(rule, layout, word_bits, planes_a, planes_b, X, Y, t0, steps, choice["k"],
                            choice.get("tile_rows", 0), stream, row_loop=choice.get("loop", 0),
                            words_per_lane=choice.get("width", 0))


def tune(rule, layout: int, word_bits: int, planes_a, planes_b, X: int, Y: int, candidates=DEFAULT_CANDIDATES,
         burst_steps: int = 48, use_cache: bool = True) -> dict:
    """Measure each candidate (mode, k[, tile_rows]) on (planes_a, planes_b) and
    return the fastest.

    The planes are used as scratch: their content after tuning is some
    evolution of the input.  Returns {"mode", "k", "tile_rows", "ns_per_cell_step"}.
    """
    import torch

    rule = lib.rule_id(rule)
    dev = torch.cuda.get_device_name(torch.cuda.current_device())
    key = _key(rule, layout, word_bits, X, Y, dev)
    if use_cache:
        with _lock:
            if key in _memo:
                return _memo[key]
            disk = _load_file().get(key)
            if disk:
                _memo[key] = disk
                return disk
    best = None
    stream = torch.cuda.current_stream().cuda_stream
    for cand in candidates:
        mode, k = cand[0], cand[1]
        th = cand[2] if len(cand) > 2 else 0
        loop = cand[3] if len(cand) > 3 else 0
        width = cand[4] if len(cand) > 4 else 0
        if th and th - 2 * ((k + 7) // 8 * 8) < 8:
            continue  # the halos would leave no interior
        if width == 2 and lib.rule_planes(rule) > 3:
            continue  # these rules have only the one-word-per-lane kernel
        choice = {"mode": mode, "k": k, "tile_rows": th, "loop": loop, "width": width}
        steps = max(burst_steps, 2 * k) // k * k
        try:
            run(choice, rule, layout, word_bits, planes_a, planes_b, X, Y, 0, k, stream)  # warm-up
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run(choice, rule, layout, word_bits, planes_a, planes_b, X, Y, 0, steps, stream)
            e1.record()
            e1.synchronize()
        except lib.CellatoError:
            continue
        ns = e0.elapsed_time(e1) * 1e6 / (X * Y * steps)
        if best is None or ns < best["ns_per_cell_step"]:
            best = dict(choice, ns_per_cell_step=ns)
    if best is None:
        raise RuntimeError("no autotune candidate ran")
    if use_cache:
        with _lock:
            _memo[key] = best
        _store_file(key, best)
    return best
