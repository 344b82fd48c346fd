"""Whole-grid operations and the simulation server on the device.

* cellato_checksum: the reference's 4 x 4 tile sums of state values, computed
  from the planes, against the oracle's checksum of the unpacked cells, over
  every rule, layout and word size, with widths whose words straddle tile
  columns and heights that do not divide by four.
* cellato_fill_random: the device generator against a numpy restatement of
  its defining formula.
* cellato_server_*: requests of all ten automata, mixed sizes and step counts,
  submitted in waves while iterations run, under a tile budget that keeps only
  part of them active at a time.  Every result -- planes and checksum -- equals
  the same grid run alone through cellato_run_temporal with the same k, and the
  small ones equal the oracle.  Admission under a tight memory cap keeps the
  resident bytes within the cap.
All of it is integer bitwise work: comparisons are exact."""
import numpy as np
import pytest

from cellato_b200 import inputs, lib

from conftest import RULES

pytestmark = pytest.mark.gpu

def splitmix_cells(seed, X, Y, thresholds):
    """numpy restatement of cellato_fill_random's cell indices."""
    n = np.arange(X * Y, dtype=np.uint64).reshape(Y, X)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (n + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(32)).astype(np.uint64)
    idx = np.zeros((Y, X), dtype=np.uint8)
    for t in thresholds:
        idx += (u >= np.uint64(t)).astype(np.uint8)
    return idx


def device_checksum(rule, layout, W, ptrs, X, Y):
    import torch
    sums = torch.zeros(16, dtype=torch.int64, device="cuda")
    lib.checksum(rule, layout, W, ptrs, X, Y, sums.data_ptr())
    torch.cuda.synchronize()
    return [int(v) & 0xFFFFFFFFFFFFFFFF for v in sums.cpu().tolist()]


LAYOUTS = [(0, 32), (0, 64), (1, 32), (1, 64)]


@pytest.mark.parametrize("layout,W", LAYOUTS)
def test_checksum_matches_oracle(cuda, oracle, layout, W):
    from cellato_b200.device import DevicePlanes
    rng = np.random.default_rng(11 + layout * 7 + W)
    R = W // 8 if layout == 1 else 1
    shapes = [(64, 64), (128, 40), (192, 8 * R), (320, 72)] if W == 64 else [(32, 16), (96, 40), (160, 24), (64, 72)]
    for r in range(10):
        for X, Y in shapes:
            if layout == 1 and Y % R:
                continue
            cells = rng.integers(0, inputs.STATES[r], size=(Y, X), dtype=np.uint8)
            nb = inputs.PLANES[r]
            a = DevicePlanes(nb, X, Y)
            a.upload(oracle.pack(layout, W, nb, cells))
            got = lib.checksum_string(device_checksum(r, layout, W, a.ptrs, X, Y))
            assert got == oracle.checksum(r, cells), (RULES[r], layout, W, X, Y)


def test_checksum_large_grid_against_numpy(cuda, oracle):
    """A 4096 x 4096 grid of the 32-state automaton (five planes), against tile
    sums of the state values taken with numpy."""
    from cellato_b200.device import DevicePlanes
    X, Y = 4096, 4096
    rng = np.random.default_rng(5)
    r = 6  # cyclic: 32 states, 5 planes
    cells = rng.integers(0, 32, size=(Y, X), dtype=np.uint8)
    a = DevicePlanes(5, X, Y)
    a.upload(oracle.pack(1, 64, 5, cells))
    sums = device_checksum(r, 1, 64, a.ptrs, X, Y)
    values = np.array([lib.state_value(r, i) for i in range(32)], dtype=np.int64)
    tiles = values[cells].reshape(4, Y // 4, 4, X // 4).sum(axis=(1, 3))
    assert sums == [int(v) for v in tiles.reshape(-1)]


@pytest.mark.parametrize("layout,W", LAYOUTS)
def test_fill_random_matches_formula(cuda, oracle, layout, W):
    from cellato_b200.device import DevicePlanes
    for r, (X, Y) in [(2, (256, 64)), (6, (128, 48)), (1, (64, 16)), (3, (192, 40))]:
        th = inputs.thresholds(inputs.REFERENCE_DENSITY[RULES[r]])
        nb = inputs.PLANES[r]
        a = DevicePlanes(nb, X, Y)
        lib.fill_random(layout, W, nb, a.ptrs, X, Y, 1234 + r, th)
        got = oracle.unpack(layout, W, nb, a.download(), X, Y)
        assert np.array_equal(got, splitmix_cells(1234 + r, X, Y, th)), (RULES[r], layout, W)


def test_fill_random_density(cuda):
    from cellato_b200.device import DevicePlanes
    X = Y = 1024
    probs = inputs.REFERENCE_DENSITY["wire"]
    a = DevicePlanes(2, X, Y)
    lib.fill_random(1, 64, 2, a.ptrs, X, Y, 99, inputs.thresholds(probs))
    cells = a.unpack(1, 64).cpu().numpy()
    freq = np.bincount(cells.reshape(-1), minlength=4) / cells.size
    for i, p in probs.items():
        assert abs(freq[i] - p) < 0.005, (i, freq[i], p)


def alone(rule, layout, W, X, Y, steps, k, seed, th):
    """The same request run by itself: fill, then the single-grid traverser."""
    from cellato_b200.device import DevicePlanes
    nb = inputs.PLANES[rule]
    a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
    lib.fill_random(layout, W, nb, a.ptrs, X, Y, seed, th)
    init = a.download()
    in_b = lib.run_temporal(rule, layout, W, a.ptrs, b.ptrs, X, Y, 0, steps, k)
    res = b if in_b else a
    return init, res.download(), device_checksum(rule, layout, W, res.ptrs, X, Y)


@pytest.mark.parametrize("layout,W", [(1, 64), (0, 32)])
def test_server_mix_matches_runs_alone(cuda, oracle, layout, W):
    from cellato_b200.serve import Server
    rng = np.random.default_rng(21 + layout)
    ks = {r: [3, 5, 8, 4, 6, 7, 2, 5, 4, 6][r] for r in range(10)}
    R = W // 8 if layout == 1 else 1
    reqs = []
    for i in range(60):
        r = i % 10
        X = int(rng.integers(1, 9)) * 64
        Y = int(rng.integers(1, 40)) * 8
        Y -= Y % R
        steps = 0 if i % 17 == 0 else int(rng.integers(1, 120))
        th = inputs.thresholds(inputs.REFERENCE_DENSITY[RULES[r]])
        reqs.append((r, X, Y, steps, 1000 + i, th))
    done = {}
    with Server(layout, W, tile_budget=12, chunk_rounds=2, k_per_rule=ks) as srv:
        ids = {}
        waves = [reqs[0:20], reqs[20:35], reqs[35:60]]
        for wave in waves:
            for q in wave:
                r, X, Y, steps, seed, th = q
                ids[srv.submit_random(r, X, Y, steps, seed, thresholds=th, keep=True)] = q
            for _ in range(3):  # some iterations before the next wave arrives
                srv.iterate()
                for res in srv.poll():
                    done[res["id"]] = res
        for res in srv.run_until_idle():
            done[res["id"]] = res
        assert sorted(done) == sorted(ids)
        st = srv.stats()
        assert st["iterations"] > 3 and st["running"] == 0 and st["waiting"] == 0
        for rid, (r, X, Y, steps, seed, th) in ids.items():
            res = done[rid]
            nb = inputs.PLANES[r]
            served = lib.download_planes(nb, srv.planes(rid, nb), X * Y // 8)
            init, ref, ref_sum = alone(r, layout, W, X, Y, steps, ks[r], seed, th)
            assert np.array_equal(served, ref), (rid, RULES[r], X, Y, steps)
            assert res["checksum"] == ref_sum, rid
            if X * Y * max(steps, 1) <= 64 * 64 * 120:
                cells = oracle.unpack(layout, W, nb, init, X, Y)
                want = oracle.run(r, cells, steps)
                assert np.array_equal(oracle.unpack(layout, W, nb, served, X, Y), want), (rid, RULES[r])
            srv.release(rid)
        assert srv.stats()["resident_bytes"] == 0


def test_server_admission_cap_and_host_planes(cuda, oracle):
    from cellato_b200.serve import Server
    rng = np.random.default_rng(8)
    layout, W = 1, 64
    X, Y = 256, 128
    per_request = 2 * 2 * ((X * Y // 8 + 255) // 256 * 256)   # two buffers of 2 planes
    cap = 3 * per_request
    reqs = []
    with Server(layout, W, hbm_cap_bytes=cap, k_per_rule={2: 6}) as srv:
        for i in range(12):
            cells = rng.integers(0, 4, size=(Y, X), dtype=np.uint8)
            planes = oracle.pack(layout, W, 2, cells)
            steps = int(rng.integers(1, 50))
            rid = srv.submit_planes("wire", X, Y, steps, [planes[0], planes[1]])
            reqs.append((rid, cells, steps))
        results = {}
        while srv.pending():
            srv.iterate()
            st = srv.stats()
            assert st["resident_bytes"] <= cap, st
            for res in srv.poll():
                results[res["id"]] = res
        for rid, cells, steps in reqs:
            want = oracle.checksum(2, oracle.run(2, cells, steps))
            assert lib.checksum_string(results[rid]["checksum"]) == want, rid


def test_server_rejects_bad_requests(cuda):
    from cellato_b200.serve import Server
    with Server(1, 64) as srv:
        with pytest.raises(lib.CellatoError):
            srv.submit_random(42, 64, 64, 10, 1)
        with pytest.raises(lib.CellatoError):
            srv.submit_random("wire", 100, 64, 10, 1)       # X not a multiple of 32
        with pytest.raises(lib.CellatoError):
            srv.submit_random("wire", 64, 12, 10, 1)        # Y not a multiple of 8
        with pytest.raises(lib.CellatoError):
            srv.submit_random("wire", 64, 64, -1, 1)
        with pytest.raises(lib.CellatoError):
            srv.submit_random("wire", 64, 64, 10, 1, thresholds=[5, 3])   # descending
        with pytest.raises(lib.CellatoError):
            srv.submit_random("game-of-life", 64, 64, 10, 1, thresholds=[1, 2])  # 3 indices, 1 plane
        with pytest.raises(lib.CellatoError):
            srv.release(12345)
        assert srv.iterate() == 0


def test_server_snapshot_cancel_resume(cuda, oracle):
    """Preemption without recomputation: requests are advanced part-way, then
    checkpointed (planes + steps done + next step number) and cancelled, and
    resumed on a second server from the snapshot with the steps left.  The
    rules whose steps alternate (traffic, critters' Margolus phase) are among
    them and resume from odd step numbers.  Results equal the uninterrupted
    run alone; a snapshot of a request that keeps running leaves its result
    unchanged."""
    from cellato_b200.serve import Server
    layout, W = 1, 64
    ks = {r: 3 for r in range(10)}      # odd k: snapshots fall on odd step numbers
    reqs = [(9, 128, 64, 40), (8, 192, 48, 31), (3, 256, 64, 25), (6, 64, 32, 17), (2, 128, 128, 45),
            (0, 64, 64, 9)]
    with Server(layout, W, chunk_rounds=1, k_per_rule=ks) as a, Server(layout, W, k_per_rule=ks) as b:
        ids = []
        for i, (r, X, Y, steps) in enumerate(reqs):
            th = inputs.thresholds(inputs.REFERENCE_DENSITY[RULES[r]])
            ids.append(a.submit_random(r, X, Y, steps, 500 + i, thresholds=th, keep=True))
        a.iterate()                     # one round of 3 steps each
        resumed, kept_running = {}, None
        for i, rid in enumerate(ids):
            r, X, Y, steps = reqs[i]
            nb = inputs.PLANES[r]
            planes, done, nxt = a.snapshot(rid, nb, X, Y)
            assert nxt == done and 0 < done < steps, (i, done, nxt)
            if i == len(ids) - 1:
                kept_running = rid   # this one is checkpointed but left to run on
                continue
            a.cancel(rid)
            resumed[b.submit_planes(r, X, Y, steps - done, list(planes), keep=True, t0=nxt)] = i
        results = {res["id"]: res for res in b.run_until_idle()}
        results.update({res["id"]: res for res in a.run_until_idle()})
        for rid, i in list(resumed.items()) + [(kept_running, len(ids) - 1)]:
            r, X, Y, steps = reqs[i]
            srv = a if rid == kept_running else b
            nb = inputs.PLANES[r]
            got = lib.download_planes(nb, srv.planes(rid, nb), X * Y // 8)
            th = inputs.thresholds(inputs.REFERENCE_DENSITY[RULES[r]])
            init, ref, ref_sum = alone(r, layout, W, X, Y, steps, ks[r], 500 + i, th)
            assert np.array_equal(got, ref), (i, RULES[r])
            assert results[rid]["checksum"] == ref_sum, i
            cells = oracle.unpack(layout, W, nb, init, X, Y)
            assert np.array_equal(oracle.unpack(layout, W, nb, got, X, Y), oracle.run(r, cells, steps)), i
        with pytest.raises(lib.CellatoError):
            a.snapshot(ids[0], 1, 128, 64)    # cancelled: nothing held


def test_diff_cells(cuda, oracle):
    """Full-grid diff against numpy on unpacked cells, for each layout and plane
    count, on grids whose plane size is and is not a multiple of 16 bytes."""
    import torch
    from cellato_b200.device import DevicePlanes
    rng = np.random.default_rng(31)
    for layout, W in LAYOUTS:
        for r, (X, Y) in [(6, (4096, 512)), (2, (64, 8)), (0, (32, 9)), (7, (96, 40))]:
            if (layout == 1 and Y % (W // 8)) or (layout == 0 and X % W):
                continue
            nb = inputs.PLANES[r]
            c1 = rng.integers(0, inputs.STATES[r], size=(Y, X), dtype=np.uint8)
            c2 = c1.copy()
            flips = rng.random((Y, X)) < 0.01
            c2[flips] = (c2[flips] + 1) % inputs.STATES[r]
            a, b = DevicePlanes(nb, X, Y), DevicePlanes(nb, X, Y)
            a.upload(oracle.pack(layout, W, nb, c1))
            b.upload(oracle.pack(layout, W, nb, c2))
            out = torch.zeros(1, dtype=torch.int64, device="cuda")
            lib.diff_cells(nb, a.ptrs, b.ptrs, X * Y // 8, out.data_ptr())
            torch.cuda.synchronize()
            assert int(out.item()) == int((c1 != c2).sum()), (layout, W, RULES[r], X, Y)
            lib.diff_cells(nb, a.ptrs, a.ptrs, X * Y // 8, out.data_ptr())
            torch.cuda.synchronize()
            assert int(out.item()) == 0
