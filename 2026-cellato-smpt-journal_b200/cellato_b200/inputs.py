"""Seeded synthetic initial grids.

There is no public dataset behind this hot path: the reference only ever runs
seeded random grids (src/<automaton>/data_init.hpp, drawn with std::mt19937 and
a cumulative-threshold walk in include/memory/grid_utils.hpp:15-57).  These
generators draw the distributions the benchmark workloads name, with numpy's
PCG64 and the same cumulative-threshold rule ("first state whose cumulative
probability is >= r").  Cells are returned as uint8 *dictionary indices* --
the integer the bit planes encode -- in a (Y, X) array.

Large grids are drawn in row chunks so that host memory stays bounded.
"""
from __future__ import annotations

import numpy as np

RULES = ["game-of-life", "forest-fire", "wire", "excitable", "brian",
         "maze", "cyclic", "fluid", "critters", "traffic"]
RULE_ID = {n: i for i, n in enumerate(RULES)}
RULE_ID["fire"] = 1

PLANES = [1, 2, 2, 3, 2, 1, 5, 4, 1, 2]
STATES = [2, 4, 4, 8, 3, 2, 32, 16, 2, 3]

# Each automaton's reference density (src/<a>/data_init.hpp), as dictionary
# index -> probability.  wire's reference initialiser draws a structured circuit
# rather than i.i.d. cells; the i.i.d. mix named for the WireWorld workload
# (empty/conductor/head/tail = .50/.40/.05/.05) stands in for it.
REFERENCE_DENSITY = {
    "game-of-life": {0: 0.8, 1: 0.2},
    "forest-fire": {0: 0.20, 1: 0.79, 2: 0.01, 3: 0.0},
    "wire": {0: 0.50, 3: 0.40, 1: 0.05, 2: 0.05},
    "excitable": {0: 0.70, 1: 0.15, 2: 0.05, 3: 0.03, 4: 0.03, 5: 0.02, 6: 0.01, 7: 0.01},
    "brian": {0: 0.8, 2: 0.2},
    "maze": {0: 0.8, 1: 0.2},
    "cyclic": {i: 1.0 / 32 for i in range(32)},
    "fluid": {i: 1.0 / 16 for i in range(16)},
    "critters": {0: 0.5, 1: 0.5},
    "traffic": {0: 0.5, 1: 0.25, 2: 0.25},
}


def categorical(X: int, Y: int, probs: dict, seed: int, chunk_rows: int = 1024) -> np.ndarray:
    """i.i.d. cells: index i with probability probs[i] (cumulative thresholds)."""
    items = list(probs.items())
    cum = np.cumsum([p for _, p in items])
    vals = np.array([s for s, _ in items], dtype=np.uint8)
    out = np.empty((Y, X), dtype=np.uint8)
    rng = np.random.Generator(np.random.PCG64(seed))
    for y0 in range(0, Y, chunk_rows):
        y1 = min(Y, y0 + chunk_rows)
        r = rng.random((y1 - y0, X))
        k = np.searchsorted(cum, r, side="left")
        np.minimum(k, len(vals) - 1, out=k)
        out[y0:y1] = vals[k]
    return out


def bernoulli_bits(X: int, Y: int, nbits: int, p: float, seed: int, chunk_rows: int = 1024) -> np.ndarray:
    """Each of the low `nbits` bits of every cell set i.i.d. with probability p."""
    out = np.zeros((Y, X), dtype=np.uint8)
    rng = np.random.Generator(np.random.PCG64(seed))
    for y0 in range(0, Y, chunk_rows):
        y1 = min(Y, y0 + chunk_rows)
        acc = np.zeros((y1 - y0, X), dtype=np.uint8)
        for b in range(nbits):
            acc |= (rng.random((y1 - y0, X)) < p).astype(np.uint8) << b
        out[y0:y1] = acc
    return out


def uniform(X: int, Y: int, n_states: int, seed: int) -> np.ndarray:
    return categorical(X, Y, {i: 1.0 / n_states for i in range(n_states)}, seed)


def workload_grid(name: str, X: int, Y: int, seed: int) -> np.ndarray:
    """The initial grid of a named benchmark workload.

    * game-of-life: Bernoulli(0.5) alive
    * wire: i.i.d. empty/conductor/head/tail = .50/.40/.05/.05
    * excitable (Greenberg-Hastings): uniform over its 8 states
    * cyclic: uniform over its 32 states
    * fluid (HPP): each of the 4 direction bits set i.i.d. with p = 0.3
    * anything else: the automaton's reference density
    """
    if name == "game-of-life":
        return categorical(X, Y, {0: 0.5, 1: 0.5}, seed)
    if name == "wire":
        return categorical(X, Y, REFERENCE_DENSITY["wire"], seed)
    if name == "excitable":
        return uniform(X, Y, 8, seed)
    if name == "cyclic":
        return uniform(X, Y, 32, seed)
    if name == "fluid":
        return bernoulli_bits(X, Y, 4, 0.3, seed)
    return categorical(X, Y, REFERENCE_DENSITY[name], seed)


def reference_density_grid(name: str, X: int, Y: int, seed: int) -> np.ndarray:
    return categorical(X, Y, REFERENCE_DENSITY[name], seed)


def thresholds(probs: dict) -> list:
    """Thresholds of the device generator (cellato_fill_random) for index
    probabilities {index: p}: t_i = floor(P(index <= i) * 2^32) for i below the
    last index with p > 0, so that index = #{i : t_i <= u} for a uniform u32."""
    last = max(i for i, p in probs.items() if p > 0)
    out, cum = [], 0.0
    for i in range(last):
        cum += probs.get(i, 0.0)
        out.append(min(int(cum * 2.0 ** 32), 2 ** 32 - 1))
    return out
