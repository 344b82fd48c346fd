"""The rule lowering (b200/lower.cuh, including the compile-time LOP3
synthesis) compiled for the host and run over linear plane words, against the
golden fixtures -- a CPU check of the same templates the sm_100a kernels use."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT, RULES

SRC = os.path.join(ROOT, "tests", "cpp", "host_lowering.cpp")


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("hl") / "libhost_lowering.so")
    subprocess.run(["g++", "-std=c++20", "-O2", "-fPIC", "-shared", f"-I{PKG}/include", f"-I{PKG}/automata",
                    "-o", out, SRC], check=True)
    lib = ctypes.CDLL(out)
    u8 = ctypes.POINTER(ctypes.c_uint8)
    lib.host_lowered_run.argtypes = [ctypes.c_int, u8, u8] + [ctypes.c_int] * 4
    lib.host_config_init.argtypes = [ctypes.c_int] * 4 + [u8]
    return lib


def run(lib, rule, cells, steps, t0=0):
    cells = np.ascontiguousarray(cells)
    out = np.empty_like(cells)
    u8 = ctypes.POINTER(ctypes.c_uint8)
    Y, X = cells.shape
    assert lib.host_lowered_run(rule, cells.ctypes.data_as(u8), out.ctypes.data_as(u8), X, Y, t0, steps) == 0
    return out


def test_lowering_matches_golden(host_lib, golden_small):
    for case, cin, cout in golden_small:
        assert np.array_equal(run(host_lib, RULES.index(case["rule"]), cin, case["steps"]), cout), case["key"]


def test_lowering_step_offsets(host_lib, oracle):
    rng = np.random.default_rng(3)
    for r in range(10):
        cells = rng.integers(0, oracle.states(r), (48, 96), dtype=np.uint8)
        for t0 in (1, 4, 7):
            assert np.array_equal(run(host_lib, r, cells, 7, t0), oracle.run(r, cells, 7, t0=t0)), (RULES[r], t0)


def test_config_initialisers_match_reference(host_lib):
    """Every automaton's seeded initial grid (config::input::random, what the
    cellato CLI starts from) equals the reference's own initialiser for the
    same seed -- WireWorld's structured circuit included."""
    import oracle as oracle_mod
    try:
        ref = oracle_mod.RefOracle()
    except FileNotFoundError:
        pytest.skip("reference build not present")
    u8 = ctypes.POINTER(ctypes.c_uint8)
    for r in range(10):
        for X, Y, seed in [(256, 128, 7), (64, 64, 1), (320, 96, 12345), (1024, 512, 42), (96, 40, 3)]:
            got = np.empty((Y, X), dtype=np.uint8)
            assert host_lib.host_config_init(r, X, Y, seed, got.ctypes.data_as(u8)) == 0
            want = ref.reference_init(r, X, Y, seed)
            assert np.array_equal(got, want), (RULES[r], X, Y, seed, int((got != want).sum()))
