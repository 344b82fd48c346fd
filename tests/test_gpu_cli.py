"""The C++ drop-in layer end to end on the GPU: the `cellato` CLI (reference
flags, suite selection and CSV line) over the grid / traverser shims and the C
ABI, checked like the reference's verify.py -- its 4x4 tile checksum must equal
the reference CPU standard path's on the reference's own seeded initial grid."""
import os
import subprocess

import pytest

from conftest import PKG, RULES

pytestmark = pytest.mark.gpu

CLI = os.path.join(PKG, "bin", "cellato")
HEADER = None


def run_cli(args):
    r = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip().splitlines()[-1]


@pytest.mark.parametrize("traverser,layout,word", [("simple", "bit_planes", 64), ("simple", "tiled_bit_planes", 32),
                                                   ("temporal", "bit_planes", 32), ("temporal", "tiled_bit_planes", 64)])
def test_cli_checksums_match_reference(cuda, traverser, layout, word):
    from oracle import RefOracle
    ref = RefOracle()
    header = run_cli(["--print_csv_header"]).split(",")
    X, Y, steps, seed = 256, 128, 24, 7
    for rule, name in enumerate(RULES):
        args = ["--automaton", name, "--device", "CUDA", "--traverser", traverser, "--evaluator", layout,
                "--layout", layout, "--word_size", str(word), "--x_size", str(X), "--y_size", str(Y),
                "--steps", str(steps), "--seed", str(seed), "--rounds", "2"]
        if traverser == "temporal":
            args += ["--temporal_steps", "4"]
        row = dict(zip(header, run_cli(args).split(",")))
        cells = ref.reference_init(rule, X, Y, seed)
        want = ref.checksum(rule, ref.run_standard(rule, cells, steps))
        assert row["checksum"] == want, (name, traverser, layout, word)
        assert row["rounds_had_same_checksums"] == "true"


def test_cli_rejects_unknown_suite_and_reports_bad_sizes(cuda):
    r = subprocess.run([CLI, "--automaton", "game-of-life", "--device", "CPU", "--traverser", "simple",
                        "--evaluator", "standard", "--layout", "standard", "--word_size", "64",
                        "--x_size", "64", "--y_size", "8", "--steps", "1"], capture_output=True, text=True)
    assert r.returncode == 2 and "No suitable test suite" in r.stderr
    r = subprocess.run([CLI, "--automaton", "game-of-life", "--device", "CUDA", "--traverser", "simple",
                        "--evaluator", "bit_planes", "--layout", "bit_planes", "--word_size", "64",
                        "--x_size", "96", "--y_size", "8", "--steps", "1"], capture_output=True, text=True)
    assert r.returncode == 3


@pytest.mark.parametrize("word,X", [(32, 480), (64, 1344)])
def test_cli_bit_array_checksums_match_reference(cuda, word, X):
    """The reference's bit_array suite (--evaluator bit_array --layout bit_array,
    the simple traverser): a bit_array grid built from the reference's seeded
    state, converted to planes on the device, stepped, converted back.  The widths
    are multiples of 32 and of every rule's cells per word."""
    from oracle import RefOracle
    ref = RefOracle()
    header = run_cli(["--print_csv_header"]).split(",")
    Y, steps, seed = 40, 17, 11
    for rule, name in enumerate(RULES):
        args = ["--automaton", name, "--device", "CUDA", "--traverser", "simple", "--evaluator", "bit_array",
                "--layout", "bit_array", "--word_size", str(word), "--x_size", str(X), "--y_size", str(Y),
                "--steps", str(steps), "--seed", str(seed), "--rounds", "2"]
        row = dict(zip(header, run_cli(args).split(",")))
        cells = ref.reference_init(rule, X, Y, seed)
        want = ref.checksum(rule, ref.run_standard(rule, cells, steps))
        assert row["checksum"] == want, (name, word)
        assert row["rounds_had_same_checksums"] == "true"
