"""bench.py's host logic on the CPU: pinned choices, the text a choice is
reported as, and the gating of ncu-derived constants by the hash of the
kernel sources they were captured from."""
import importlib.util
import os
import sys

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    argv = sys.argv
    sys.argv = ["bench.py"]
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_parse_choices(bench):
    got = bench.parse_choices("wire=temporal:16:0:3:1:32,excitable=temporal:8:128:2,brian=simple_stream")
    assert got["wire"] == {"mode": "temporal", "k": 16, "tile_rows": 0, "loop": 3, "width": 1, "word_bits": 32}
    assert got["excitable"] == {"mode": "temporal", "k": 8, "tile_rows": 128, "loop": 2, "width": 0}
    assert got["brian"] == {"mode": "simple_stream", "k": 1, "tile_rows": 0}
    assert bench.parse_choices("") == {}


def test_describe_choice(bench):
    assert bench.describe_choice({"mode": "temporal", "k": 16, "tile_rows": 0, "loop": 3, "width": 1,
                                  "word_bits": 32}) == "temporal k=16 tile_rows=0 loop=paired words_per_lane=1 W32"
    assert bench.describe_choice({"mode": "simple_tma", "k": 1, "width": 4}) == "simple_tma words_per_lane=4"
    assert bench.describe_choice({"mode": "simple_register", "k": 1}) == "simple_register"


def test_measured_constants_are_gated_by_the_kernel_source_hash(bench):
    h = bench.kernel_source_hash("wire")
    assert len(h) == 16 and h == bench.kernel_source_hash("wire")
    assert h != bench.kernel_source_hash("cyclic")  # the rule's own headers enter the hash
    table = {("wire", 1): (5.0, "profiles/x.md", h), ("wire", 2): (6.0, "profiles/x.md", "0" * 16),
             ("wire", 3): (7.0, "profiles/x.md", None)}
    assert bench.measured(table, ("wire", 1), "wire") == (5.0, "profiles/x.md", True)
    assert bench.measured(table, ("wire", 2), "wire")[2] is False
    assert bench.measured(table, ("wire", 3), "wire")[2] is False
    assert bench.measured(table, ("wire", 4), "wire") is None


def test_committed_captures_name_their_sources(bench):
    """Every ncu-derived constant in bench.py names the profile summary it
    comes from and the hash of the kernel sources it was captured from."""
    for table in (bench.MEASURED_TRAFFIC, bench.MEASURED_ALU):
        for key, (value, src, digest) in table.items():
            assert value > 0 and key[0] in bench.AUTOMATON_DIRS, key
            assert os.path.exists(os.path.join(ROOT, src)), src
            assert isinstance(digest, str) and len(digest) == 16, key
