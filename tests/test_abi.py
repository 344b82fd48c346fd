"""The C-ABI library: loads, exports every symbol include/cellato_b200.h
declares, and validates arguments on the host (no GPU needed for these paths)."""
import ctypes
import os
import re

import pytest

from cellato_b200 import inputs, lib

from conftest import ROOT, RULES


def declared_functions():
    text = open(os.path.join(ROOT, "include", "cellato_b200.h")).read()
    return sorted(set(re.findall(r"\b(cellato_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = lib.load()
    names = declared_functions()
    assert names, "no declarations parsed"
    assert sorted(lib.EXPORTED) == names
    for n in names:
        assert hasattr(L, n), n


def test_version():
    assert lib.load().cellato_version().decode().startswith("cellato-b200")


def test_rule_table_matches_reference_dictionaries():
    for r, name in enumerate(RULES):
        assert lib.rule_id(name) == r
        assert lib.rule_name(r) == name
        assert lib.rule_planes(r) == inputs.PLANES[r]
        assert lib.rule_states(r) == inputs.STATES[r]
    assert lib.rule_id("fire") == 1
    assert lib.load().cellato_rule_from_name(b"no-such-rule") == -1


@pytest.mark.parametrize("layout,W,X,Y,ok", [
    (0, 32, 32, 1, True), (0, 64, 64, 3, True), (0, 64, 96, 8, False), (0, 32, 48, 8, False),
    (1, 32, 32, 4, True), (1, 32, 32, 6, False), (1, 64, 64, 8, True), (1, 64, 64, 12, False),
    (0, 16, 64, 8, False), (2, 32, 64, 8, False), (0, 32, 0, 8, False),
])
def test_check_dims(layout, W, X, Y, ok):
    rc = lib.load().cellato_check_dims(layout, W, X, Y)
    assert (rc == lib.OK) == ok, (rc, lib.load().cellato_last_error())


def test_plane_bytes():
    assert lib.load().cellato_plane_bytes(2048, 2048) == 2048 * 2048 // 8
    assert lib.load().cellato_plane_bytes(0, 5) == 0


def test_run_rejects_bad_arguments_before_touching_the_device():
    a = [0x1000, 0x2000]
    b = [0x3000, 0x4000]
    with pytest.raises(lib.CellatoError) as e:
        lib.run_simple("wire", 0, 64, a, b, 96, 8, 0, 1)
    assert e.value.status == lib.EINVAL_DIMS
    with pytest.raises(lib.CellatoError) as e:
        lib.run_simple("wire", 0, 64, [0x1001, 0x2000], b, 64, 8, 0, 1)
    assert e.value.status == lib.EINVAL
    with pytest.raises(lib.CellatoError) as e:
        lib.run_simple("wire", 0, 64, a, a, 64, 8, 0, 1)
    assert e.value.status == lib.EINVAL
    with pytest.raises(lib.CellatoError) as e:
        lib.run_simple(42, 0, 64, a, b, 64, 8, 0, 1)
    assert e.value.status == lib.EINVAL
    with pytest.raises(lib.CellatoError) as e:
        lib.run_temporal("wire", 0, 64, a, b, 64, 8, 0, 4, k=0)
    assert e.value.status == lib.EINVAL
    with pytest.raises(lib.CellatoError) as e:
        lib.run_temporal("wire", 0, 64, a, b, 64, 8, 0, 4, k=33)
    assert e.value.status == lib.EINVAL
    with pytest.raises(lib.CellatoError) as e:
        lib.run_simple("wire", 0, 64, a, b, 64, 8, 0, -1)
    assert e.value.status == lib.EINVAL
    # zero steps is a no-op that never launches
    assert lib.run_simple("wire", 0, 64, a, b, 64, 8, 0, 0) == 0
