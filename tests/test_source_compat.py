"""Source compatibility of the rule DSL: the reference's own automaton headers
compile unchanged against this library's header tree and, lowered by the B200
lowering (host build), reproduce the golden results."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT, RULES

# the reference tree (its src/ holds the automaton headers); override with CELLATO_REFERENCE_DIR
REF_SRC = os.path.join(os.environ.get("CELLATO_REFERENCE_DIR", "/root/reference"), "src")
SRC = os.path.join(ROOT, "tests", "cpp", "source_compat.cpp")

pytestmark = pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference source tree not present")


@pytest.fixture(scope="module")
def compat_lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("sc") / "libsource_compat.so")
    cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-w",
           f"-I{PKG}/include", f"-I{ROOT}/include", "-I/usr/local/cuda/include", f"-I{REF_SRC}",
           "-o", out, SRC]
    subprocess.run(cmd, check=True)
    lib = ctypes.CDLL(out)
    u8 = ctypes.POINTER(ctypes.c_uint8)
    lib.reference_rules_lowered_run.argtypes = [ctypes.c_int, u8, u8] + [ctypes.c_int] * 3
    return lib


def test_reference_rule_headers_compile_and_match(compat_lib, golden_small):
    u8 = ctypes.POINTER(ctypes.c_uint8)
    for case, cin, cout in golden_small:
        cin = np.ascontiguousarray(cin)
        out = np.empty_like(cin)
        Y, X = cin.shape
        rc = compat_lib.reference_rules_lowered_run(RULES.index(case["rule"]), cin.ctypes.data_as(u8),
                                                     out.ctypes.data_as(u8), X, Y, case["steps"])
        assert rc == 0
        assert np.array_equal(out, cout), case["key"]
