"""Simulation server over the C ABI cellato_server_* (continuous batching).

    srv = Server(layout=1, word_bits=64, k_per_rule={r: 16 for r in range(10)})
    rid = srv.submit_random("wire", 2048, 2048, steps=1000, seed=7,
                            probs=inputs.REFERENCE_DENSITY["wire"])
    while srv.pending():
        srv.iterate()
        for res in srv.poll():
            ...   # res["checksum"] (16 tile sums), res["done_s"] - res["submit_s"]

The server keeps each request's planes on the device from admission to
completion, admits by plane footprint (strict FIFO under hbm_cap_bytes), and
advances every active request by a chunk of rounds per iteration, one batched
launch per automaton and round.  Requests submitted with keep=True leave their
final planes on the device (planes(id)) until release(id).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import inputs, lib


class Server:
    def __init__(self, layout: int = 1, word_bits: int = 64, hbm_cap_bytes: int = 0, tile_budget: int = 0,
                 chunk_rounds: int = 0, max_inflight: int = 0, k_per_rule=None):
        L = lib.load()
        cfg = lib.ServerConfig()
        cfg.layout, cfg.word_bits = layout, word_bits
        cfg.hbm_cap_bytes = hbm_cap_bytes
        cfg.tile_budget, cfg.chunk_rounds, cfg.max_inflight = tile_budget, chunk_rounds, max_inflight
        self._ks, cfg.n_k_per_rule = lib.k_array(k_per_rule)  # the array outlives the create call
        cfg.k_per_rule = self._ks
        h = ctypes.c_void_p()
        lib.check(L.cellato_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.layout, self.word_bits = layout, word_bits
        self._outstanding = 0
        self._buf = (lib.ServerResult * 256)()

    # -- submission
    def submit_random(self, rule, X: int, Y: int, steps: int, seed: int, probs=None, thresholds=None,
                      keep: bool = False) -> int:
        """A request whose initial state is the device generator's draw
        (cellato_fill_random) from `seed` with index probabilities `probs`
        ({index: p}) or explicit `thresholds`."""
        rule = lib.rule_id(rule)
        if thresholds is None:
            thresholds = inputs.thresholds(probs) if probs is not None else []
        th = (ctypes.c_uint32 * max(1, len(thresholds)))(*thresholds)
        rid = ctypes.c_longlong()
        lib.check(lib.load().cellato_server_submit_random(self._h, rule, X, Y, steps, seed, th, len(thresholds),
                                                          int(keep), ctypes.byref(rid)))
        self._outstanding += 1
        return rid.value

    def submit_planes(self, rule, X: int, Y: int, steps: int, host_planes, keep: bool = False,
                      t0: int = 0) -> int:
        """A request whose initial state is given as host planes (numpy arrays,
        one per plane, in the server's layout), its first step numbered t0
        (a snapshot's next_step when resuming)."""
        rule = lib.rule_id(rule)
        arrs = [np.ascontiguousarray(p) for p in host_planes]
        ptrs = (ctypes.c_void_p * max(1, len(arrs)))(*[a.ctypes.data for a in arrs])
        rid = ctypes.c_longlong()
        lib.check(lib.load().cellato_server_submit_resume(self._h, rule, X, Y, steps, t0, ptrs, int(keep),
                                                          ctypes.byref(rid)))
        self._outstanding += 1
        return rid.value

    def snapshot(self, rid: int, nb: int, X: int, Y: int):
        """Checkpoint of a request: (planes as an (nb, X*Y/8) uint8 array,
        steps done, next step number).  The request keeps running."""
        out = np.empty((nb, X * Y // 8), dtype=np.uint8)
        ptrs = (ctypes.c_void_p * 8)(*[out[p].ctypes.data for p in range(nb)])
        done, nxt = ctypes.c_int(), ctypes.c_int()
        lib.check(lib.load().cellato_server_snapshot(self._h, rid, ptrs, ctypes.byref(done), ctypes.byref(nxt)))
        return out, done.value, nxt.value

    def cancel(self, rid: int, completed: bool = False) -> None:
        """Removes a request and frees its planes (pass completed=True for a
        kept request whose result poll() already returned)."""
        lib.check(lib.load().cellato_server_cancel(self._h, rid))
        if not completed:
            self._outstanding -= 1

    # -- progress
    def iterate(self) -> int:
        """One scheduling iteration; returns the number of requests it advanced."""
        n = ctypes.c_int()
        lib.check(lib.load().cellato_server_iterate(self._h, ctypes.byref(n)))
        return n.value

    def poll(self):
        """Completed requests since the last poll, as dicts."""
        out = []
        n = ctypes.c_int()
        while True:
            lib.check(lib.load().cellato_server_poll(self._h, self._buf, len(self._buf), ctypes.byref(n)))
            for i in range(n.value):
                r = self._buf[i]
                out.append({"id": r.id, "rule": r.rule, "x": r.x_cells, "y": r.y_cells, "steps": r.steps,
                            "result_in_b": r.result_in_b, "checksum": [int(v) for v in r.checksum],
                            "submit_s": r.submit_s, "done_s": r.done_s})
            if n.value < len(self._buf):
                break
        self._outstanding -= len(out)
        return out

    def pending(self) -> int:
        """Requests submitted and not yet returned by poll()."""
        return self._outstanding

    def run_until_idle(self):
        """Iterates until every submitted request has completed; returns them."""
        done = []
        while self._outstanding:
            self.iterate()
            done.extend(self.poll())
        return done

    # -- results kept on the device
    def planes(self, rid: int, nb: int):
        arr = (ctypes.c_void_p * 8)()
        lib.check(lib.load().cellato_server_planes(self._h, rid, arr))
        return [arr[p] for p in range(nb)]

    def release(self, rid: int) -> None:
        lib.check(lib.load().cellato_server_release(self._h, rid))

    def stats(self) -> dict:
        st = lib.ServerStats()
        lib.check(lib.load().cellato_server_stats_get(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in lib.ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            lib.load().cellato_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
