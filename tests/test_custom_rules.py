"""Rules outside the library (the header-only custom-rule path).

tests/cpp/custom_rules.hpp writes three automata that neither the reference
nor this library ships in the rule DSL.  tests/cpp/custom_rules_gpu.cu
instantiates them outside the library from the package's public headers
(b200/custom_rule.cuh); the tests hand the tables to cellato_rule_register and
run them through the C ABI.  The expected grids (tests/golden/custom.npz) are
the reference's own standard evaluator run on the same rule source
(oracle/_ref/libcellato_ref_custom.so), and a numpy restatement below pins them
a second way.
"""
import ctypes
import json
import os
import threading
import time

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

CUSTOM_LIB = os.path.join(ROOT, "tests", "cpp", "_build", "libcustom_rules.so")
LAYOUTS = [(0, 32), (0, 64), (1, 32), (1, 64)]
PLANES = {"highlife": 1, "star-wars": 2, "parity-shift": 1}


@pytest.fixture(scope="module")
def custom_cases():
    d = np.load(os.path.join(GOLDEN, "custom.npz"))
    index = json.loads(bytes(d["index"]).decode())
    return [(c, d[c["key"] + "_in"], d[c["key"] + "_out"]) for c in index]


@pytest.fixture(scope="module")
def custom_ids():
    """Registers the three custom rules; returns {name: rule id}."""
    from cellato_b200 import lib
    so = ctypes.CDLL(CUSTOM_LIB)
    so.custom_rule_table.restype = ctypes.c_void_p
    so.custom_rule_table.argtypes = [ctypes.c_int]
    ids = {}
    for which in range(so.custom_rule_count()):
        rid = lib.rule_register(so.custom_rule_table(which))
        ids[lib.rule_name(rid)] = rid
    ids["_so"] = so
    return ids


# ---- numpy restatement of the three rules (test infrastructure) -----------
def _moore(a):
    return sum(np.roll(np.roll(a, dy, 0), dx, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if dy or dx)


def numpy_run(rule, cells, steps):
    c = cells.astype(np.int64)
    for t in range(steps):
        if rule == "highlife":
            n = _moore(c == 1)
            c = np.where(c == 1, (n == 2) | (n == 3), (n == 3) | (n == 6)).astype(np.int64)
        elif rule == "star-wars":
            n = _moore(c == 1)
            c = np.select([c == 1, c == 2, c == 3], [np.where((n > 2) & (n < 6), 1, 2), 3, 0],
                          np.where(n == 2, 1, 0))
        else:  # parity-shift: parity on even steps, shift right on odd ones
            if t % 2 == 0:
                on = c == 1
                n = np.roll(on, 1, 0).astype(int) + np.roll(on, -1, 0) + np.roll(on, 1, 1) + np.roll(on, -1, 1)
                c = (n % 2 == 1).astype(np.int64)
            else:
                c = np.roll(c, 1, 1)
    return c.astype(np.uint8)


def test_custom_fixtures_match_numpy_restatement(custom_cases):
    for case, cin, cout in custom_cases:
        assert np.array_equal(numpy_run(case["rule"], cin, case["steps"]), cout), case["key"]


def test_custom_fixtures_match_reference_evaluator(custom_cases):
    import oracle as oracle_mod
    try:
        ref = oracle_mod.RefCustomOracle()
    except FileNotFoundError:
        pytest.skip("reference custom-rule build not present")
    for case, cin, cout in custom_cases:
        assert np.array_equal(ref.run_standard(case["which"], cin, case["steps"]), cout), case["key"]


def test_register_custom_rules(custom_ids):
    """Registration needs no GPU: ids follow the built-in ones, names resolve,
    a second registration of a table returns its id, and tables with a
    duplicate name or another rule_ops layout are refused."""
    from cellato_b200 import lib
    L = lib.load()
    so = custom_ids["_so"]
    for name, planes in PLANES.items():
        rid = custom_ids[name]
        assert rid >= lib.BUILTIN_RULES
        assert lib.rule_id(name) == rid
        assert lib.rule_planes(rid) == planes
        assert lib.rule_register(so.custom_rule_table(["highlife", "star-wars", "parity-shift"].index(name))) == rid
    assert lib.rule_count() >= lib.BUILTIN_RULES + 3
    # a copy of a table under the same name, and one claiming another layout
    src = so.custom_rule_table(0)
    size = ctypes.c_int.from_address(src + 4).value
    buf = (ctypes.c_char * size).from_buffer_copy((ctypes.c_char * size).from_address(src))
    out = ctypes.c_int(-1)
    assert L.cellato_rule_register(ctypes.addressof(buf), ctypes.byref(out)) == lib.EINVAL
    assert b"already registered" in L.cellato_last_error()
    ctypes.c_int.from_buffer(buf, 0).value = 999
    assert L.cellato_rule_register(ctypes.addressof(buf), ctypes.byref(out)) == lib.EINVAL
    assert b"ABI" in L.cellato_last_error()


def _run(rule, layout, W, cells, steps, mode, k=1, t0=0, **tune):
    import torch
    from cellato_b200 import lib
    from cellato_b200.device import DevicePlanes
    import oracle as oracle_mod
    o = oracle_mod.Oracle()
    Y, X = cells.shape
    nb = lib.rule_planes(rule)
    a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
    a.upload(o.pack(layout, W, nb, cells))
    if mode == "simple":
        in_b = lib.run_simple(rule, layout, W, a.ptrs, b.ptrs, X, Y, t0, steps, **tune)
    else:
        in_b = lib.run_temporal(rule, layout, W, a.ptrs, b.ptrs, X, Y, t0, steps, k, **tune)
    torch.cuda.synchronize()
    return o.unpack(layout, W, nb, (b if in_b else a).download(), X, Y)


@pytest.mark.gpu
@pytest.mark.parametrize("layout,W", LAYOUTS)
def test_custom_rules_on_gpu_match_reference(cuda, custom_ids, custom_cases, layout, W):
    """Single-step kernels (both) and the temporal kernel (k = 1, 3, 5, 8, 16,
    the three row loops and both widths) on the custom rules against the
    reference."""
    runs = [("simple", 1, {}), ("simple", 1, {"simple_kernel": 2}), ("temporal", 1, {}), ("temporal", 3, {}),
            ("temporal", 8, {"row_loop": 1, "words_per_lane": 2}), ("temporal", 16, {"row_loop": 2}),
            ("temporal", 5, {"row_loop": 3}), ("temporal", 8, {"row_loop": 3, "words_per_lane": 2})]
    for case, cin, cout in custom_cases:
        rid = custom_ids[case["rule"]]
        for mode, k, tune in runs:
            got = _run(rid, layout, W, cin, case["steps"], mode, k, **tune)
            assert np.array_equal(got, cout), (case["key"], mode, k, tune)


@pytest.mark.gpu
def test_custom_rule_in_a_batch_with_builtin_rules(cuda, custom_ids, custom_cases):
    """A batch that mixes custom and built-in rules equals each grid run alone."""
    import torch
    from cellato_b200 import inputs, lib
    from cellato_b200.batch import Batch
    from cellato_b200.device import DevicePlanes
    rng = np.random.default_rng(5)
    specs = [(custom_ids["highlife"], 256, 64, 33), (custom_ids["star-wars"], 192, 48, 50),
             (custom_ids["parity-shift"], 128, 32, 17), (lib.rule_id("wire"), 256, 64, 40),
             (lib.rule_id("critters"), 128, 32, 21)]
    grids, want = [], []
    for rule, X, Y, steps in specs:
        nb, n = lib.rule_planes(rule), lib.rule_states(rule)
        a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
        lib.fill_random(1, 64, nb, a.ptrs, X, Y, int(rng.integers(1 << 30)),
                        inputs.thresholds({i: 1.0 / n for i in range(n)}))
        ra, rb = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
        ra.buf.copy_(a.buf)
        in_b = lib.run_temporal(rule, 1, 64, ra.ptrs, rb.ptrs, X, Y, 0, steps, 6)
        torch.cuda.synchronize()
        want.append((rb if in_b else ra).download())
        grids.append((a, b))
    ks = {rule: 6 for rule, _, _, _ in specs}
    batch = Batch(1, 64, [(r, X, Y, s, a.ptrs, b.ptrs) for (r, X, Y, s), (a, b) in zip(specs, grids)], ks)
    batch.launch()
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(grids):
        got = (b if batch.result_in_b(i) else a).download()
        assert np.array_equal(got, want[i]), (i, specs[i])


@pytest.mark.gpu
def test_two_threads_two_streams_different_tunings(cuda):
    """Per-call tuning has no shared state: two host threads drive two streams
    with different kernels, row loops and tile widths at once, repeatedly, and
    each gets the result of its own configuration run alone."""
    import torch
    from cellato_b200 import inputs, lib
    from cellato_b200.device import DevicePlanes
    X, Y, steps = 2048, 512, 48
    rule = lib.rule_id("excitable")
    nb = lib.rule_planes(rule)
    tunings = [("simple", 1, {"simple_kernel": 1}), ("simple", 1, {"simple_kernel": 2}),
               ("temporal", 8, {"row_loop": 1, "words_per_lane": 2, "tile_rows": 64}),
               ("temporal", 8, {"row_loop": 2, "words_per_lane": 1})]
    init = DevicePlanes(nb, X, Y)
    lib.fill_random(0, 64, nb, init.ptrs, X, Y, 99, inputs.thresholds(inputs.REFERENCE_DENSITY["excitable"]))
    torch.cuda.synchronize()
    # the expected grid, one configuration alone
    a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
    a.buf.copy_(init.buf)
    in_b = lib.run_simple(rule, 0, 64, a.ptrs, b.ptrs, X, Y, 0, steps)
    torch.cuda.synchronize()
    want = (b if in_b else a).download()

    errors = []

    def worker(pair):
        try:
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):  # allocated and zeroed on the thread's own stream
                bufs = [(DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)) for _ in pair]
            for _ in range(6):
                for (mode, k, tune), (pa, pb) in zip(pair, bufs):
                    with torch.cuda.stream(st):
                        pa.buf.copy_(init.buf)
                    if mode == "simple":
                        f = lib.run_simple(rule, 0, 64, pa.ptrs, pb.ptrs, X, Y, 0, steps, st.cuda_stream, **tune)
                    else:
                        f = lib.run_temporal(rule, 0, 64, pa.ptrs, pb.ptrs, X, Y, 0, steps, k,
                                             stream=st.cuda_stream, **tune)
                    st.synchronize()
                    got = (pb if f else pa).download()
                    if not np.array_equal(got, want):
                        errors.append((mode, k, tune))
        except Exception as e:  # surfaced below
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=(tunings[:2],)),
               threading.Thread(target=worker, args=(tunings[2:],))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors


@pytest.mark.gpu
def test_batch_wait_that_runs_out_returns_and_counts(cuda, custom_ids):
    """Failure handling of the persistent batch kernel's bounded waits, with
    no device fault: an item waits for a round that is never run (a count that
    nothing raises).  The wait gives up after its poll limit, the launch
    returns, the timeout is counted, and the device stays usable."""
    import torch
    so = custom_ids["_so"]
    so.custom_batch_wait_probe.argtypes = [ctypes.c_uint, ctypes.POINTER(ctypes.c_uint)]
    n = ctypes.c_uint(99)
    t = time.perf_counter()
    assert so.custom_batch_wait_probe(4096, ctypes.byref(n)) == 0
    assert time.perf_counter() - t < 10.0
    assert n.value == 1
    x = torch.arange(1024, device="cuda")
    assert int(x.sum()) == 1024 * 1023 // 2
