"""The autotuner's host logic (candidate filter, tie rule, cache keys and file)
on the CPU, and on the GPU that its pick is reproducible and that the word size
is a tuning dimension."""
import json

import pytest

from cellato_b200 import autotune, lib


def test_legal_candidates_filter():
    cands = [("simple_register", 1), ("temporal", 8, 0, 2, 2), ("temporal", 24, 48, 1, 1),
             ("temporal", 24, 80, 1, 1), ("temporal", 16, 320, 2, 1), ("temporal", 16, 192, 2, 2)]
    # a five-plane rule: no two-words-per-lane tile; 48 rows leave no interior at k = 24 (R = 8)
    got = autotune.legal_candidates(cands, planes=5, band_rows=8)
    assert [(c["mode"], c["k"], c["tile_rows"], c["width"]) for c in got] == [
        ("simple_register", 1, 0, 0), ("temporal", 24, 80, 1), ("temporal", 16, 320, 1)]
    # a two-plane rule keeps width 2; shared memory limits drop the tallest tiles
    got = autotune.legal_candidates(cands, planes=2, max_tile_rows={0: 256, 1: 256, 2: 128}, band_rows=8)
    assert [(c["k"], c["tile_rows"], c["width"]) for c in got] == [(1, 0, 0), (8, 0, 2), (24, 80, 1)]
    # the linear layout (R = 1): the halo is k rows
    got = autotune.legal_candidates([("temporal", 24, 56, 1, 1)], planes=1, band_rows=1)
    assert got and got[0]["tile_rows"] == 56
    assert autotune.legal_candidates([("temporal", 24, 48, 1, 1)], planes=1, band_rows=1) == []


def test_candidate_sets_cover_widths_and_row_loops():
    """TMA widths 1, 2, 4 as single-step candidates, four words per lane only
    for one-plane rules; the three row loops among the temporal candidates."""
    tma = [c for c in autotune.SINGLE_STEP_CANDIDATES if c[0] == "simple_tma"]
    assert {c[4] for c in tma if len(c) > 4} == {1, 2, 4}
    widths = lambda planes: sorted({c["width"] for c in autotune.legal_candidates(tma, planes=planes)})
    assert widths(1) == [0, 1, 2, 4] and widths(2) == [0, 1, 2] and widths(5) == [0, 1]
    loops = {c[3] for c in autotune.DEFAULT_CANDIDATES if c[0] == "temporal" and len(c) > 3}
    assert loops == {1, 2, 3}
    # two steps per sweep at k = 1 would be the hoisted loop: not a candidate
    assert not [c for c in autotune.DEFAULT_CANDIDATES if c[0] == "temporal" and c[1] == 1 and len(c) > 3
                and c[3] == 3]


def test_pick_takes_the_earliest_within_the_tie_band():
    a, b, c = {"k": 1}, {"k": 8}, {"k": 16}
    assert autotune.pick([(a, 1.00), (b, 0.99), (c, 0.90)])["k"] == 16
    assert autotune.pick([(a, 1.00), (b, 0.99), (c, 0.985)])["k"] == 1
    assert autotune.pick([(a, 1.10), (b, 1.00), (c, 1.015)])["k"] == 8
    assert autotune.pick([]) is None


def test_cache_keys(tmp_path):
    k = autotune.cache_key(2, 1, 64, 16384, 16384, "B200", "abc")
    assert k == autotune.cache_key(2, 1, 64, 16384, 16000, "B200", "abc")  # same size class
    others = [autotune.cache_key(2, 1, 64, 16384, 16384, "B200", "abd"),
              autotune.cache_key(3, 1, 64, 16384, 16384, "B200", "abc"),
              autotune.cache_key(2, 0, 64, 16384, 16384, "B200", "abc"),
              autotune.cache_key(2, 1, 32, 16384, 16384, "B200", "abc"),
              autotune.cache_key(2, 1, 64, 32768, 32768, "B200", "abc"),
              autotune.cache_key(2, 1, 64, 16384, 16384, "H100", "abc"),
              autotune.cache_key(2, 1, 64, 16384, 16384, "B200", "abc", candidates=[("temporal", 8)])]
    assert k not in others and len(set(others)) == len(others)
    # the build id follows the library file's bytes
    f1, f2 = tmp_path / "a.so", tmp_path / "b.so"
    f1.write_bytes(b"one build")
    f2.write_bytes(b"another build")
    assert autotune.build_id(str(f1)) != autotune.build_id(str(f2))
    assert autotune.build_id(str(f1)) == autotune.build_id(str(f1))
    assert len(autotune.build_id()) == 16


def test_cache_file_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("CELLATO_AUTOTUNE_CACHE", str(path))
    autotune._store_file("k1", {"mode": "temporal", "k": 8})
    autotune._store_file("k2", {"mode": "simple_stream", "k": 1})
    assert json.loads(path.read_text()) == {"k1": {"mode": "temporal", "k": 8},
                                            "k2": {"mode": "simple_stream", "k": 1}}
    assert autotune._load_file()["k2"]["mode"] == "simple_stream"
    path.write_text("not json")
    assert autotune._load_file() == {}


@pytest.mark.gpu
def test_pick_is_reproducible_and_word_size_is_tuned(cuda):
    import torch
    from cellato_b200 import inputs
    from cellato_b200.device import DevicePlanes
    X = Y = 4096
    rule = lib.rule_id("wire")
    nb = lib.rule_planes(rule)
    cands = (("simple_register", 1), ("temporal", 1, 128, 2, 1), ("temporal", 8, 0, 2, 1),
             ("temporal", 16, 0, 2, 1), ("temporal", 16, 0, 1, 2))
    picks = []
    for _ in range(2):
        a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
        lib.fill_random(1, 64, nb, a.ptrs, X, Y, 5, inputs.thresholds(inputs.REFERENCE_DENSITY["wire"]))
        c = autotune.tune(rule, 1, 64, a.ptrs, b.ptrs, X, Y, candidates=cands, use_cache=False)
        picks.append({n: c[n] for n in ("mode", "k", "tile_rows", "loop", "width")})
    assert picks[0] == picks[1]
    cells = torch.from_numpy(inputs.workload_grid("wire", X, Y, 5)).cuda()
    c = autotune.tune_word_bits(rule, 1, cells, X, Y, candidates=cands, use_cache=False)
    assert c["word_bits"] in (32, 64) and c["mode"] in ("simple_register", "temporal")
