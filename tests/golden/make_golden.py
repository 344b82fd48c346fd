"""Generate the golden fixtures from the reference's own CPU code.

Run where the reference tree is present (it builds oracle/_ref first):

    make -C oracle && python tests/golden/make_golden.py

Every expected output here comes from the *reference* CPU standard path
(evaluators::standard + traversers::cpu::simple, compiled from the reference
headers into oracle/_ref/libcellato_ref.so).  The fixtures pin both the C
restatement in oracle/ and the GPU path.

* small.npz   -- full input/output grids (uint8 dictionary indices) for small
                 cases of every automaton: uniform random states, the
                 reference's own seeded initialiser, odd step counts, one-word
                 wide and ragged shapes.
* large.json  -- workload-sized cases stored as SHA-256 of the input and output
                 grids plus the reference 4x4 tile checksum string; the input is
                 regenerated from the named seeded generator and its hash checked.
* custom.npz  -- full input/output grids of the three custom rules of
                 tests/cpp/custom_rules.hpp (rules outside the reference and the
                 library), run by the reference's standard path instantiated for
                 them (oracle/_ref/libcellato_ref_custom.so).

`python tests/golden/make_golden.py custom` writes custom.npz alone.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "2026-cellato-smpt-journal_b200"))

from oracle import RefCustomOracle, RefOracle  # noqa: E402
from cellato_b200 import inputs  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint8).tobytes()).hexdigest()


# (generator, X, Y, steps, seed)
SMALL_CASES = [
    ("uniform", 128, 64, 37, 100),
    ("reference_init", 256, 128, 64, 42),
    ("workload", 64, 16, 1, 7),
    ("workload", 192, 24, 10, 8),
    ("uniform", 64, 8, 9, 9),
    ("reference_density", 256, 256, 100, 11),
    ("uniform", 384, 48, 23, 12),
]

# (rule, generator, X, Y, steps, seed, note)
LARGE_CASES = [
    ("game-of-life", "workload", 2048, 2048, 100, 42, "GoL 2048^2 Bernoulli(0.5), 100 steps"),
    ("wire", "workload", 2048, 2048, 1000, 42, "WireWorld 2048^2 crop of the 16384^2 workload"),
    ("excitable", "workload", 2048, 2048, 1000, 42, "Greenberg-Hastings 2048^2 crop of the 16384^2 workload"),
    ("cyclic", "workload", 4096, 4096, 256, 42, "cyclic 4096^2 crop of the 32768^2 workload"),
    ("fluid", "workload", 4096, 4096, 256, 42, "HPP fluid 4096^2 crop of the 32768^2 workload"),
    ("forest-fire", "reference_density", 1024, 1024, 200, 5, "forest fire 1024^2"),
    ("brian", "reference_density", 1024, 1024, 200, 5, "Brian's brain 1024^2"),
    ("maze", "reference_density", 1024, 1024, 200, 5, "maze 1024^2"),
    ("critters", "reference_density", 1024, 1024, 200, 5, "critters 1024^2"),
    ("traffic", "reference_density", 1024, 1024, 201, 5, "traffic 1024^2, odd steps"),
]


def make_input(ref: RefOracle, rule: int, gen: str, X: int, Y: int, seed: int) -> np.ndarray:
    name = inputs.RULES[rule]
    if gen == "uniform":
        return inputs.uniform(X, Y, inputs.STATES[rule], seed)
    if gen == "reference_init":
        return ref.reference_init(rule, X, Y, seed)
    if gen == "workload":
        return inputs.workload_grid(name, X, Y, seed)
    if gen == "reference_density":
        return inputs.reference_density_grid(name, X, Y, seed)
    raise ValueError(gen)


# (X, Y, steps, seed) for the custom rules: uniform random states
CUSTOM_CASES = [(64, 8, 9, 1), (128, 64, 37, 2), (192, 24, 64, 3), (256, 256, 100, 4), (320, 48, 23, 5)]


def make_custom() -> None:
    ref = RefCustomOracle()
    arrays, index = {}, []
    for which in range(ref.count()):
        for ci, (X, Y, steps, seed) in enumerate(CUSTOM_CASES):
            cells = inputs.uniform(X, Y, ref.states(which), 1000 * which + seed)
            key = f"c{which}_{ci}"
            arrays[key + "_in"] = cells
            arrays[key + "_out"] = ref.run_standard(which, cells, steps)
            index.append({"key": key, "rule": ref.name(which), "which": which, "X": X, "Y": Y, "steps": steps,
                          "seed": 1000 * which + seed})
    arrays["index"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "custom.npz"), **arrays)
    print(f"custom.npz: {len(index)} cases")


def main() -> None:
    if sys.argv[1:] == ["custom"]:
        make_custom()
        return
    make_custom()
    ref = RefOracle()
    threads = os.cpu_count() or 1
    arrays = {}
    index = []
    for rule, name in enumerate(inputs.RULES):
        for ci, (gen, X, Y, steps, seed) in enumerate(SMALL_CASES):
            cells = make_input(ref, rule, gen, X, Y, seed)
            out = ref.run_standard(rule, cells, steps)
            key = f"r{rule}_c{ci}"
            arrays[key + "_in"] = cells
            arrays[key + "_out"] = out
            index.append({"key": key, "rule": name, "generator": gen, "X": X, "Y": Y,
                          "steps": steps, "seed": seed, "checksum": ref.checksum(rule, out)})
    arrays["index"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "small.npz"), **arrays)
    print(f"small.npz: {len(index)} cases")

    large = []
    for name, gen, X, Y, steps, seed, note in LARGE_CASES:
        rule = inputs.RULE_ID[name]
        cells = make_input(ref, rule, gen, X, Y, seed)
        t = time.time()
        out = ref.run_standard(rule, cells, steps, threads=threads)
        dt = time.time() - t
        large.append({"rule": name, "generator": gen, "X": X, "Y": Y, "steps": steps, "seed": seed,
                      "note": note, "sha256_in": sha(cells), "sha256_out": sha(out),
                      "checksum": ref.checksum(rule, out)})
        print(f"{name} {X}x{Y}x{steps}: {dt:.1f}s on {threads} threads")
    meta = {"generated_by": "tests/golden/make_golden.py",
            "oracle": "reference CPU standard path (evaluators::standard + traversers::cpu::simple)",
            "cases": large}
    with open(os.path.join(HERE, "large.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
