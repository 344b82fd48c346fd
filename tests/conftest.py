import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "2026-cellato-smpt-journal_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
RULES = ["game-of-life", "forest-fire", "wire", "excitable", "brian",
         "maze", "cyclic", "fluid", "critters", "traffic"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    lib = os.path.join(PKG, "lib", "libcellato_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-j8", "-C", PKG], check=True, capture_output=True)
    # rebuilt when its sources or the package headers changed (make's own check)
    subprocess.run(["make", "-C", os.path.join(ROOT, "tests", "cpp")], check=True, capture_output=True)
    olib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(olib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden_small():
    d = np.load(os.path.join(GOLDEN, "small.npz"))
    index = json.loads(bytes(d["index"]).decode())
    return [(c, d[c["key"] + "_in"], d[c["key"] + "_out"]) for c in index]


@pytest.fixture(scope="session")
def golden_large():
    with open(os.path.join(GOLDEN, "large.json")) as f:
        return json.load(f)["cases"]


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
