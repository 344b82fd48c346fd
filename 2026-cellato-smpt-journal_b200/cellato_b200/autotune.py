"""Autotuner: picks the traverser configuration per automaton and grid size.

The reference leaves (temporal_steps, temporal_tile_size_y, cuda_block_size_y)
to the user and sweeps them with run_all.py (src/_scripts/cluster_run/
run_all.py:9-24).  Here the choice is measured on the device: each candidate --
a single-step kernel, or the temporal kernel with k fused steps at a tile
height, row loop and tile width -- runs bursts on the caller's own device
planes; the median of the bursts is its time per cell-step.  Every choice is
passed to the library per call (cellato_tune), so tuning never changes what
other callers run.

Reproducibility: candidates within TIE_BAND of the fastest count as ties, and
the earliest of them in candidate order wins, so run-to-run noise does not flip
the pick between near-equal configurations.

Word width: for the tiled layout the word size sets the tile height in rows (4
for 32-bit words, 8 for 64-bit ones), which the caller may leave open;
tune_word_bits packs the grid both ways and tunes each.  For the linear layout
32- and 64-bit words are the same bytes and the same kernels.

Results are cached per (library build, rule, layout, word size, size class,
device) in memory and in a JSON file, so a server or batch launcher pays the
search once; a rebuilt library never reuses an older build's picks.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import statistics
import threading

from . import lib

# (mode, k[, tile_rows[, row loop[, words per lane]]]); tile_rows 0 = the
# library's default height for k; row loop as cellato_tune.row_loop (1 row by
# row, 2 hoisted, 3 two steps per sweep) and words
# per lane as cellato_tune.words_per_lane (0 = default; two words per lane exist
# only for rules of up to three planes, four only for one-plane rules, and are
# skipped for the others; for simple_tma the width is the TMA kernel's words per
# lane).
# Single-step candidates: the single-step kernels and the temporal kernel at
# k = 1 (one step per launch through a shared-memory tile), which for rules with
# many planes or long networks reaches more of the HBM roofline.
SINGLE_STEP_CANDIDATES = (("simple_register", 1), ("simple_stream", 1), ("simple_tma", 1)) + tuple(
    ("simple_tma", 1, 0, 0, width) for width in (1, 2, 4)) + tuple(
    ("temporal", 1, th, loop, width) for th in (0, 96, 128, 192) for loop in (1, 2) for width in (1, 2))
DEFAULT_CANDIDATES = SINGLE_STEP_CANDIDATES + (("temporal", 2), ("temporal", 2, 0, 3)) + tuple(
    ("temporal", k, th, loop, width) for k in (4, 6, 8, 12, 16, 24) for th in (0, 96, 128, 160, 192, 256, 320)
    for loop in (1, 2, 3) for width in (1, 2))
_VARIANT = {"simple": 0, "simple_register": 1, "simple_stream": 2, "simple_tma": 3}

TIE_BAND = 0.02   # candidates within 2% of the fastest are ties
REPEATS = 3       # timed bursts per candidate (the median counts)

_lock = threading.Lock()
_memo: dict = {}
_build_id = None


def size_class(X: int, Y: int) -> int:
    """log2 of the cell count, rounded: grids within a factor ~1.4 share a tuning."""
    return int(round(math.log2(max(1, X * Y))))


def cache_path() -> str:
    return os.environ.get("CELLATO_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "cellato_b200_autotune.json"))


def build_id(path: str | None = None) -> str:
    """First 16 hex digits of the SHA-256 of the library file: picks cached for
    one build are not reused by another."""
    global _build_id
    if path is None and _build_id is not None:
        return _build_id
    h = hashlib.sha256()
    with open(path or lib.LIB_PATH, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    digest = h.hexdigest()[:16]
    if path is None:
        _build_id = digest
    return digest


def cache_key(rule: int, layout: int, word_bits: int, X: int, Y: int, device_name: str, build: str,
              candidates=None) -> str:
    """Key of a tuning: the build, the problem (rule, layout, word size, size
    class), the device and, when it is not the default set, the candidate set."""
    cand = "" if candidates in (None, DEFAULT_CANDIDATES) else "/" + hashlib.sha256(
        repr(tuple(candidates)).encode()).hexdigest()[:8]
    return f"v9/{build}/{rule}/{layout}/{word_bits}/{size_class(X, Y)}/{device_name}{cand}"


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


def legal_candidates(candidates, planes: int, max_tile_rows: dict | None = None, band_rows: int = 8):
    """The candidates a rule of `planes` planes can run, as choice dicts:
    two words per lane only for rules of up to three planes; a fixed tile
    height must leave interior rows below both halos (ceil(k/R)*R rows each,
    R = band_rows) and fit in shared memory (max_tile_rows: {words per lane:
    tallest tile}, when known)."""
    out = []
    for cand in candidates:
        mode, k = cand[0], cand[1]
        th = cand[2] if len(cand) > 2 else 0
        loop = cand[3] if len(cand) > 3 else 0
        width = cand[4] if len(cand) > 4 else 0
        if (width == 2 and planes > 3) or (width == 4 and planes > 1):
            continue
        if th:
            halo = -(-k // band_rows) * band_rows
            if th - 2 * halo < 8:
                continue
            if max_tile_rows is not None and th > max_tile_rows.get(width, th):
                continue
        out.append({"mode": mode, "k": k, "tile_rows": th, "loop": loop, "width": width})
    return out


def pick(timed):
    """timed: [(choice, ns_per_cell_step)] in candidate order -> the earliest
    candidate within TIE_BAND of the fastest (None if empty)."""
    if not timed:
        return None
    best = min(ns for _, ns in timed)
    for choice, ns in timed:
        if ns <= best * (1.0 + TIE_BAND):
            return dict(choice, ns_per_cell_step=ns)
    return None


def run(choice: dict, rule: int, layout: int, word_bits: int, planes_a, planes_b, X: int, Y: int, t0: int,
        steps: int, stream: int = 0) -> int:
    """Run `steps` steps with a tuned choice; returns 1 if the result is in planes_b."""
    if choice["mode"] in _VARIANT:
        return lib.run_simple(rule, layout, word_bits, planes_a, planes_b, X, Y, t0, steps, stream,
                              simple_kernel=_VARIANT[choice["mode"]], words_per_lane=choice.get("width", 0))
    return lib.run_temporal(rule, layout, word_bits, planes_a, planes_b, X, Y, t0, steps, choice["k"],
                            choice.get("tile_rows", 0), stream, row_loop=choice.get("loop", 0),
                            words_per_lane=choice.get("width", 0))


def tune(rule, layout: int, word_bits: int, planes_a, planes_b, X: int, Y: int, candidates=DEFAULT_CANDIDATES,
         burst_steps: int = 48, use_cache: bool = True, repeats: int = REPEATS) -> dict:
    """Measure each legal candidate on (planes_a, planes_b) and return the pick.

    The planes are used as scratch: their content after tuning is some
    evolution of the input.  Returns {"mode", "k", "tile_rows", "loop",
    "width", "ns_per_cell_step"}.
    """
    import torch

    rule = lib.rule_id(rule)
    dev = torch.cuda.get_device_name(torch.cuda.current_device())
    key = cache_key(rule, layout, word_bits, X, Y, dev, build_id(), candidates)
    if use_cache:
        with _lock:
            if key in _memo:
                return _memo[key]
            disk = _load_file().get(key)
            if disk:
                _memo[key] = disk
                return disk
    R = 1 if layout == lib.LAYOUT_BIT_PLANES else word_bits // 8
    max_rows = {w: lib.temporal_max_tile_rows(rule, layout, word_bits, w) for w in (0, 1, 2)}
    stream = torch.cuda.current_stream().cuda_stream
    timed = []
    for choice in legal_candidates(candidates, lib.rule_planes(rule), max_rows, R):
        k = choice["k"]
        steps = max(burst_steps, 2 * k) // k * k
        try:
            run(choice, rule, layout, word_bits, planes_a, planes_b, X, Y, 0, k, stream)  # warm-up
            samples = []
            for _ in range(repeats):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                run(choice, rule, layout, word_bits, planes_a, planes_b, X, Y, 0, steps, stream)
                e1.record()
                e1.synchronize()
                samples.append(e0.elapsed_time(e1) * 1e6 / (X * Y * steps))
        except lib.CellatoError:
            continue
        timed.append((choice, statistics.median(samples)))
    best = pick(timed)
    if best is None:
        raise RuntimeError("no autotune candidate ran")
    if use_cache:
        with _lock:
            _memo[key] = best
        _store_file(key, best)
    return best


def tune_word_bits(rule, layout: int, cells, X: int, Y: int, word_bits=(32, 64), candidates=DEFAULT_CANDIDATES,
                   use_cache: bool = True, **kw) -> dict:
    """The word size as a tuning dimension (where the caller allows more than
    one): packs the device grid `cells` ((Y, X) uint8 indices) into each
    allowed word size, tunes each, and returns the pick with its "word_bits".
    Word sizes the grid's shape does not allow are skipped."""
    from .device import DevicePlanes
    rule = lib.rule_id(rule)
    nb = lib.rule_planes(rule)
    timed = []
    for W in word_bits:
        if lib.load().cellato_check_dims(layout, W, X, Y) != lib.OK:
            continue
        a, b = DevicePlanes(nb, X, Y, cells.device), DevicePlanes(nb, X, Y, cells.device)
        a.pack_from(cells, layout, W)
        c = tune(rule, layout, W, a.ptrs, b.ptrs, X, Y, candidates, use_cache=use_cache, **kw)
        timed.append((dict(c, word_bits=W), c["ns_per_cell_step"]))
        del a, b
    best = pick(timed)
    if best is None:
        raise RuntimeError("no word size fits the grid")
    return best
