"""Benchmark of the B200 bit-plane hot path.

Workload (one bench step): WireWorld and Greenberg-Hastings (the `excitable`
automaton), each on one 16384 x 16384 torus in the tiled_bit_planes layout
with 64-bit words, advanced 1000 steps each; the traverser (single-step or
temporal with k fused steps) is chosen per automaton by the autotuner.
Inputs are seeded synthetic grids: WireWorld i.i.d. empty/conductor/head/tail
= .50/.40/.05/.05, Greenberg-Hastings uniform over its 8 states.

Metric: GCUPS = cell updates / s / 1e9, summed over both automata and all
ranks.  `value` times the work with the planes resident in HBM; `e2e` times the
same work through the C ABI with host buffers: every step uploads both grids'
input planes from pinned host memory, runs, and downloads the result planes.

The ping-pong plane buffers (WireWorld 128 MiB, Greenberg-Hastings 192 MiB)
exceed the 126 MB L2, so no L2 flush is inserted between steps.

The default run (--workload all) prints ONE line: the config-2 workload above
is its headline (`value`, `e2e`, rooflines, CPU baseline), and three objects
beside it carry the other workloads of the benchmark, each measured in the
same process after the previous one's memory is released:
  config3  cyclic + HPP fluid, one 32768 x 32768 bit_planes grid each, 256
           steps; GCUPS, the single-step kernels' HBM roofline and the
           temporal kernels' ALU roofline;
  batched  4096 mixed grids in one CUDA-graph launch against the same grids
           run with plain per-grid launches (ratio, bit-exactness);
  served   a Poisson request stream through the continuous-batching server
           against the same stream served one request at a time with
           per-grid launches (p50 / p99 latency, GCUPS, completed vs offered).
--workload config2|config3|batched|served prints that workload's own line.

Usage:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 run under torch.distributed.run: every rank runs the same workload on
its own GPU (replicas: the path has no exchange step) and rank 0 reports the
sum of cell updates over the maximum per-rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "2026-cellato-smpt-journal_b200")
sys.path.insert(0, PKG)

AUTOMATA = ("wire", "excitable")
SIZE = 16384
CA_STEPS = 1000
LAYOUT = 1        # tiled_bit_planes
WORD_BITS = 64
# word sizes the autotuner may pick per layout: the tiled layout's tile shape
# depends on it (8 x 4 or 8 x 8 cells); linear words of 32 and 64 bits are the
# same bytes and the same kernels, so the linear workload keeps 64
WORD_CHOICES = {0: (64,), 1: (32, 64)}
SEED = 42
BATCH_CANDIDATES = (("temporal", 2), ("temporal", 4), ("temporal", 8), ("temporal", 12), ("temporal", 16))
CPU_SAMPLE_SIZE = 2048

# DRAM bytes (read + write) per launch measured by one ncu capture of the same
# configuration (summaries in profiles/); keyed by (rule, mode, k, size).  The
# tile height and row loop change the re-read halo by about 1%, so one capture
# per k stands for them.  Each entry names the hash of the rule's kernel
# sources it was captured from (kernel_source_hash); an entry whose hash no
# longer matches the sources is reported as stale and not used.
MEASURED_TRAFFIC = {
    ("wire", "temporal", 16, 16384): (86.81e6, "profiles/temporal_kernel_dram_alu_captures.md", "99f07bc533075f2b"),
    ("excitable", "temporal", 16, 16384): (152.60e6, "profiles/temporal_kernel_dram_alu_captures.md", "c912b66d798e9644"),
    ("cyclic", "temporal", 8, 32768): (1293.47e6, "profiles/temporal_kernel_dram_alu_captures.md", "aed4cd45da7b7fcf"),
    ("fluid", "temporal", 16, 32768): (1025.98e6, "profiles/temporal_kernel_dram_alu_captures.md", "81fa5ee2a3685590"),
}

# ALU-pipe warp instructions (smsp__inst_executed_pipe_alu.sum) per launch of a
# temporal kernel configuration, from one ncu capture of that configuration
# (summary in profiles/); keyed by (rule, layout, word size, k, tile_rows, row
# loop, words per lane, size), tile_rows 0 being the library's default height.
# Each configuration is timed live and set against the ALU pipe's measured rate
# (lop3_rate) for the compute roofline.  Source hashes as above.
MEASURED_ALU = {
    ("wire", 1, 32, 16, 0, 3, 1, 16384): (111137328, "profiles/temporal_kernel_dram_alu_captures.md", "99f07bc533075f2b"),
    ("excitable", 1, 32, 16, 0, 3, 1, 16384): (71637912, "profiles/temporal_kernel_dram_alu_captures.md", "c912b66d798e9644"),
    ("cyclic", 0, 64, 8, 160, 2, 1, 32768): (813584240, "profiles/temporal_kernel_dram_alu_captures.md", "aed4cd45da7b7fcf"),
    ("fluid", 0, 64, 16, 0, 3, 1, 32768): (326666480, "profiles/temporal_kernel_dram_alu_captures.md", "81fa5ee2a3685590"),
}

AUTOMATON_DIRS = {"game-of-life": "game_of_life", "forest-fire": "fire", "wire": "wire", "excitable": "excitable",
                  "brian": "brian", "maze": "maze", "cyclic": "cyclic", "fluid": "fluid", "critters": "critters",
                  "traffic": "traffic"}


LOP3_RATE_LIB = os.path.join(ROOT, "_build", "liblop3_rate.so")


def lop3_rate(stream: int = 0) -> float:
    """Measured LOP3 lane-operations per second of the current device, the ALU
    pipe's peak for the temporal kernels' compute roofline (lop3_rate.cu, built
    by __graft_entry__.build(), or here with nvcc when that build is missing)."""
    import ctypes
    if not os.path.exists(LOP3_RATE_LIB):
        os.makedirs(os.path.dirname(LOP3_RATE_LIB), exist_ok=True)
        subprocess.run(["nvcc", "-std=c++20", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler",
                        "-fPIC", "-shared", "-o", LOP3_RATE_LIB, os.path.join(ROOT, "lop3_rate.cu"), "-lcudart"],
                       check=True)
    so = ctypes.CDLL(LOP3_RATE_LIB)
    so.lop3_rate.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    v = ctypes.c_double(0.0)
    rc = so.lop3_rate(ctypes.byref(v), stream)
    if rc != 0:
        raise RuntimeError(f"lop3_rate failed with CUDA error {rc}")
    return v.value


def kernel_source_hash(rule: str) -> str:
    """First 16 hex digits of the SHA-256 of everything a rule's kernels are
    compiled from: the lowering, the engine, the launchers, the rule's own
    headers and the build flags."""
    import hashlib
    files = [os.path.join(PKG, "include", "b200", f) for f in ("lower.cuh", "engine.cuh", "rule_kernels.cuh")]
    d = os.path.join(PKG, "automata", AUTOMATON_DIRS[rule])
    files += sorted(os.path.join(d, f) for f in os.listdir(d))
    files.append(os.path.join(PKG, "Makefile"))
    h = hashlib.sha256()
    for f in files:
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def measured(table: dict, key, rule: str):
    """(value, source, fresh) of a capture, fresh = captured from the current
    kernel sources; None when there is no capture of this configuration."""
    e = table.get(key)
    if e is None:
        return None
    value, src, digest = e
    return value, src, digest is not None and digest == kernel_source_hash(rule)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=None, help="grid side (default: the workload's)")
    ap.add_argument("--ca-steps", type=int, default=None, help="steps per automaton (default: the workload's)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sequential", action="store_true",
                    help="run the automata one after the other on one stream instead of on parallel streams")
    ap.add_argument("--choice", default="", help="pin the traverser per automaton instead of autotuning, "
                                                 "e.g. wire=temporal:8:128:1,excitable=temporal:16:0:2:1 "
                                                 "(mode:k:tile_rows:loop:words_per_lane)")
    ap.add_argument("--workload", default="all", choices=["all", "config2", "config3", "batched", "served"],
                    help="all (default): the config2 line with config3, batched and served beside it; "
                         "config2: WireWorld + Greenberg-Hastings 16384^2 x 1000 steps; "
                         "config3: cyclic + HPP fluid 32768^2 x 256 steps on bit_planes, with the single-step "
                         "kernels' HBM roofline beside the autotuned run; "
                         "batched: many mixed grids in one CUDA-graph launch vs per-grid launches; "
                         "served: a Poisson request stream through the continuous-batching server")
    ap.add_argument("--batch-grids", type=int, default=4096)
    ap.add_argument("--batch-min-side", type=int, default=64)
    ap.add_argument("--batch-max-side", type=int, default=4096)
    ap.add_argument("--batch-max-steps", type=int, default=1000)
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="length of the arrival window, s")
    ap.add_argument("--serve-min-side", type=int, default=128)
    ap.add_argument("--serve-max-side", type=int, default=8192)
    ap.add_argument("--serve-min-steps", type=int, default=100)
    ap.add_argument("--serve-max-steps", type=int, default=10000)
    ap.add_argument("--serve-check-fraction", type=float, default=0.01)
    ap.add_argument("--no-per-grid", action="store_true", help="served: skip the per-grid baseline run")
    args = ap.parse_args()
    apply_workload(args)
    return args


# workload -> (automata, side, steps per automaton, layout, largest k the
# workload's definition lets the autotuner pick)
SINGLE_GRID_WORKLOADS = {
    "config2": (("wire", "excitable"), SIZE, CA_STEPS, 1, 16),   # "temporal depth k autotuned in 1-16"
    "config3": (("cyclic", "fluid"), 32768, 256, 0, 32),
}
K_MAX = 16


def apply_workload(args, name=None) -> None:
    """Sets the automata, sizes and layout of a single-grid workload (the
    config2 ones for the batched and served workloads, whose layout and word
    size they share)."""
    global AUTOMATA, LAYOUT, K_MAX
    name = name or args.workload
    automata, side, steps, layout, kmax = SINGLE_GRID_WORKLOADS.get(name, SINGLE_GRID_WORKLOADS["config2"])
    AUTOMATA, LAYOUT, K_MAX = automata, layout, kmax
    args.size = args.size or side
    args.ca_steps = args.ca_steps or steps


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.samples = []
        if self.proc is None:
            return False
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)
        return False

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}

        def num(s):
            try:
                return float(s)
            except ValueError:
                return None

        sm = [num(s[1]) for s in self.samples if num(s[1]) is not None]
        mx = [num(s[2]) for s in self.samples if num(s[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        sm_sorted = sorted(sm)
        load = [v for v in sm_sorted if v >= 0.5 * max(sm_sorted)] if sm_sorted else []
        med = load[len(load) // 2] if load else None
        return {"sm_mhz": med, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples),
                "power_w_max": max((num(s[3]) or 0.0) for s in self.samples)}


# --------------------------------------------------------- reference arm
def load_reference_cpu():
    """The reference's own CPU path (oracle/_ref) when it was built from the
    reference tree, else the oracle's C restatement of it."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, RefOracle
    try:
        ref = RefOracle()
        return "reference", (lambda r, c, s, th: ref.run_standard(r, c, s, threads=th))
    except FileNotFoundError:
        o = Oracle()
        return "port", (lambda r, c, s, th: o.run(r, c, s, threads=th))


def cpu_sample(run, threads: int, target_s: float):
    """Time the CPU standard path on CPU_SAMPLE_SIZE^2 crops of both automata,
    sized to about target_s seconds.  Returns (GCUPS, description)."""
    from cellato_b200 import inputs
    n = CPU_SAMPLE_SIZE
    grids = {a: inputs.workload_grid(a, n, n, SEED) for a in AUTOMATA}
    t = time.perf_counter()
    for a in AUTOMATA:
        run(inputs.RULE_ID[a], grids[a], 8, threads)
    probe = time.perf_counter() - t
    steps = max(8, int(8 * 0.5 * target_s / max(probe, 1e-3)))
    # repeat bursts until the sample holds at least target_s of CPU work
    dt, total_steps = 0.0, 0
    while dt < target_s:
        t = time.perf_counter()
        for a in AUTOMATA:
            run(inputs.RULE_ID[a], grids[a], steps, threads)
        dt += time.perf_counter() - t
        total_steps += steps
    steps = total_steps
    cells = len(AUTOMATA) * n * n * steps
    return cells / dt / 1e9, f"{'+'.join(AUTOMATA)} {n}x{n} crops, {steps} steps each, {dt:.1f} s"


def reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    kind, run = load_reference_cpu()
    threads = host_threads()
    from cellato_b200 import inputs
    n = CPU_SAMPLE_SIZE
    grids = {a: inputs.workload_grid(a, n, n, SEED) for a in AUTOMATA}
    # size one step to ~4 s of work so the whole run stays within a few minutes
    t = time.perf_counter()
    for a in AUTOMATA:
        run(inputs.RULE_ID[a], grids[a], 2, threads)
    per_ca_step = (time.perf_counter() - t) / 2
    ca_steps = max(2, int(4.0 / max(per_ca_step, 1e-4)))
    for _ in range(args.warmup):
        for a in AUTOMATA:
            run(inputs.RULE_ID[a], grids[a], max(1, ca_steps // 8), threads)
    t = time.perf_counter()
    for _ in range(args.steps):
        for a in AUTOMATA:
            run(inputs.RULE_ID[a], grids[a], ca_steps, threads)
    dt = time.perf_counter() - t
    cells = args.steps * len(AUTOMATA) * n * n * ca_steps
    value = cells / dt / 1e9
    sample = f"each step: {'+'.join(AUTOMATA)} {n}x{n} crops x {ca_steps} steps, CPU standard evaluator"
    line = {
        "impl": "reference", "metric": "GCUPS", "value": round(value, 4), "unit": "GCUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": workload_config(args, extra={"cpu_sample": sample}),
        "cpu_baseline": {"value": round(value, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def parse_choices(text: str) -> dict:
    """--choice wire=temporal:8:128:1,excitable=temporal:16:0:3:1:32
    (mode:k:tile_rows:loop:words_per_lane[:word size]) or <automaton>=simple_register /
    simple_stream: pins the traverser (and the word size) per automaton."""
    out = {}
    for item in filter(None, (text or "").split(",")):
        name, spec = item.split("=")
        f = spec.split(":")
        if f[0] == "temporal":
            out[name] = {"mode": "temporal", "k": int(f[1]), "tile_rows": int(f[2]) if len(f) > 2 else 0,
                         "loop": int(f[3]) if len(f) > 3 else 0, "width": int(f[4]) if len(f) > 4 else 0}
            if len(f) > 5:
                out[name]["word_bits"] = int(f[5])
        else:
            out[name] = {"mode": f[0], "k": 1, "tile_rows": 0}
    return out


def describe_choice(c: dict) -> str:
    """The autotuner's choice as text: mode, k, tile rows (0 = default), row
    loop, tile width and, when tuned, the word size."""
    w = f" W{c['word_bits']}" if "word_bits" in c else ""
    width = {0: "default", 1: "1", 2: "2", 4: "4"}[c.get("width", 0)]
    if c["mode"] != "temporal":
        return c["mode"] + (f" words_per_lane={width}" if c.get("width", 0) else "") + w
    loop = {0: "default", 1: "row-by-row", 2: "hoisted", 3: "paired"}[c.get("loop", 0)]
    return f"temporal k={c['k']} tile_rows={c.get('tile_rows', 0)} loop={loop} words_per_lane={width}{w}"


def workload_config(args, extra=None):
    from cellato_b200 import inputs
    layout = "tiled_bit_planes" if LAYOUT == 1 else "bit_planes"
    mib = [2 * inputs.PLANES[inputs.RULE_ID[a]] * args.size * args.size // 8 >> 20 for a in AUTOMATA]
    words = "W32 or W64 autotuned" if len(WORD_CHOICES[LAYOUT]) > 1 else f"W{WORD_CHOICES[LAYOUT][0]}"
    c = {"workload": f"{'+'.join(AUTOMATA)} {args.size}x{args.size} {layout} {words}, {args.ca_steps} steps "
                     f"each, traverser autotuned (simple | temporal k <= {K_MAX})",
         "automata": list(AUTOMATA), "x_size": args.size, "y_size": args.size, "ca_steps_per_step": args.ca_steps,
         "layout": layout, "word_size": list(WORD_CHOICES[LAYOUT]),
         "l2": f"inputs larger than L2 (ping-pong planes {' MiB + '.join(str(m) for m in mib)} MiB), no flush"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------- our arm
def our_arm(args, rank: int, world: int, cpu_baseline: bool = True):
    """The single-grid workload set by apply_workload; returns its line."""
    import numpy as np
    import torch
    from cellato_b200 import autotune, inputs, lib, replicas
    from cellato_b200.device import DevicePlanes

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    X = Y = args.size
    # autotune per automaton, unless pinned: the traverser and, for the tiled
    # layout, whose word size the workload leaves open, the word size (32-bit
    # words: 8 x 4 tiles, 64-bit words: 8 x 8); then the planes in that layout
    pinned = parse_choices(args.choice)
    cands = [c for c in autotune.DEFAULT_CANDIDATES if c[1] <= K_MAX]
    grids = {}
    for a in AUTOMATA:
        r = inputs.RULE_ID[a]
        nb = inputs.PLANES[r]
        cells = torch.from_numpy(inputs.workload_grid(a, X, Y, SEED + rank)).to(dev)
        if a in pinned:
            choice = dict(pinned[a], word_bits=pinned[a].get("word_bits", WORD_BITS))
        else:
            choice = autotune.tune_word_bits(r, LAYOUT, cells, X, Y, word_bits=WORD_CHOICES[LAYOUT],
                                             candidates=cands, use_cache=False)
        W = choice["word_bits"]
        pa, pb = DevicePlanes(nb, X, Y, dev), DevicePlanes(nb, X, Y, dev)
        pa.pack_from(cells, LAYOUT, W, sp)
        init = DevicePlanes(nb, X, Y, dev)
        init.buf.copy_(pa.buf)
        del cells
        grids[a] = {"rule": r, "nb": nb, "a": pa, "b": pb, "init": init, "choice": choice, "W": W}
    torch.cuda.synchronize()

    def launches(g):
        c = g["choice"]
        return args.ca_steps if c["mode"].startswith("simple") else -(-args.ca_steps // c["k"])

    # The automata are independent grids: each runs on its own stream, forked from
    # and joined back into the timing stream, so one automaton's launches fill
    # the other's last partial wave of CTAs (--sequential runs them one after
    # the other on one stream).
    comp = {a: torch.cuda.Stream(device=dev) for a in AUTOMATA}
    fork = torch.cuda.Event()
    joins = {a: torch.cuda.Event() for a in AUTOMATA}

    def one_step(t0, events=None, concurrent=not args.sequential):
        if concurrent:
            fork.record(stream)
        for a, g in grids.items():
            st = comp[a] if concurrent else stream
            if concurrent:
                st.wait_event(fork)
            if events is not None:
                events[a][0].record(st)
            in_b = autotune.run(g["choice"], g["rule"], LAYOUT, g["W"], g["a"].ptrs, g["b"].ptrs, X, Y, t0,
                                args.ca_steps, st.cuda_stream)
            if in_b:
                g["a"], g["b"] = g["b"], g["a"]
            if events is not None:
                events[a][1].record(st)
            if concurrent:
                joins[a].record(st)
        if concurrent:
            for a in AUTOMATA:
                stream.wait_event(joins[a])

    def barrier():
        if world > 1:
            replicas.barrier()

    t0 = 0
    for _ in range(args.warmup):
        one_step(t0)
        t0 += args.ca_steps
    torch.cuda.synchronize()
    barrier()

    per = {a: [] for a in AUTOMATA}
    with ClockSampler(dev.index) as clocks:
        torch.cuda.synchronize()
        barrier()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            one_step(t0)
            t0 += args.ca_steps
        stop.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms = start.elapsed_time(stop)
    ms = max_over_ranks(ms, world)

    # each automaton alone, for its own rate and the dominant kernel's launch time
    diag_steps = 2
    for _ in range(diag_steps):
        ev = {a: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for a in AUTOMATA}
        one_step(t0, ev, concurrent=False)
        torch.cuda.synchronize()
        for a in AUTOMATA:
            per[a].append(ev[a][0].elapsed_time(ev[a][1]))
        t0 += args.ca_steps

    cells_per_step = len(AUTOMATA) * X * Y * args.ca_steps
    value = cells_per_step * args.steps * world / (ms * 1e-3) / 1e9
    per_gcups = {a: X * Y * args.ca_steps * diag_steps / (sum(per[a]) * 1e-3) / 1e9 for a in AUTOMATA}
    n_launch = sum(launches(g) for g in grids.values()) * args.steps

    # ---- end to end through the C ABI with host buffers
    host_in, host_out = {}, {}
    for a, g in grids.items():
        host_in[a] = [torch.empty(g["init"].plane_bytes, dtype=torch.uint8).pin_memory() for _ in range(g["nb"])]
        host_out[a] = [torch.empty(g["init"].plane_bytes, dtype=torch.uint8).pin_memory() for _ in range(g["nb"])]
        for p in range(g["nb"]):
            host_in[a][p].copy_(g["init"].view(p).cpu())
    h2d = sum(g["nb"] * g["init"].plane_bytes for g in grids.values())
    d2h = h2d
    L = lib.load()

    # Copies run on two copy streams, and each automaton has two device plane
    # sets used by alternate steps: a step's upload overlaps the previous
    # step's compute, and its download the next step's.  Events order each
    # set's reuse: an upload waits for the download from the same set two steps
    # earlier, the compute for its upload, the download for its compute.
    cs_in, cs_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    sets = {a: [(g["a"], g["b"]), (DevicePlanes(g["nb"], X, Y, dev), DevicePlanes(g["nb"], X, Y, dev))]
            for a, g in grids.items()}
    in_ready = {a: [torch.cuda.Event(), torch.cuda.Event()] for a in AUTOMATA}
    computed = {a: [torch.cuda.Event(), torch.cuda.Event()] for a in AUTOMATA}
    out_done = {a: [torch.cuda.Event(), torch.cuda.Event()] for a in AUTOMATA}
    start_ev = torch.cuda.Event()

    def e2e_step(i, t0):
        par = i & 1
        for a, g in grids.items():
            nb, pb_ = g["nb"], g["init"].plane_bytes
            pa, _ = sets[a][par]
            cs_in.wait_event(start_ev)
            cs_in.wait_event(out_done[a][par])
            lib.check(L.cellato_planes_upload(nb, lib.ptr_array(pa.ptrs),
                                              lib.ptr_array([t.data_ptr() for t in host_in[a]]), pb_,
                                              cs_in.cuda_stream))
            in_ready[a][par].record(cs_in)
        for a, g in grids.items():
            nb, pb_ = g["nb"], g["init"].plane_bytes
            pa, pb = sets[a][par]
            st = stream if args.sequential else comp[a]
            st.wait_event(in_ready[a][par])
            in_b = autotune.run(g["choice"], g["rule"], LAYOUT, g["W"], pa.ptrs, pb.ptrs, X, Y, t0,
                                args.ca_steps, st.cuda_stream)
            computed[a][par].record(st)
            res = pb if in_b else pa
            cs_out.wait_event(computed[a][par])
            lib.check(L.cellato_planes_download(nb, lib.ptr_array([t.data_ptr() for t in host_out[a]]),
                                                lib.ptr_array(res.ptrs), pb_, cs_out.cuda_stream))
            out_done[a][par].record(cs_out)

    for a in AUTOMATA:
        for par in (0, 1):
            out_done[a][par].record(cs_out)
    start_ev.record(stream)
    e2e_step(0, 0)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    start_ev.record(stream)
    for i in range(args.steps):
        e2e_step(i, 0)
    for a in AUTOMATA:
        for par in (0, 1):
            stream.wait_event(out_done[a][par])   # the timed region ends after the last download
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    e2e_value = cells_per_step * args.steps * world / (e2e_ms * 1e-3) / 1e9
    # the downloaded results of the last end-to-end step against a run on the device
    e2e_ok = True
    for a, g in grids.items():
        g["a"].buf.copy_(g["init"].buf)
        in_b = autotune.run(g["choice"], g["rule"], LAYOUT, g["W"], g["a"].ptrs, g["b"].ptrs, X, Y, 0,
                            args.ca_steps, sp)
        res = g["b"] if in_b else g["a"]
        torch.cuda.synchronize()
        e2e_ok &= all(torch.equal(res.view(p).cpu(), host_out[a][p]) for p in range(g["nb"]))
    del sets

    peaks = measured_peaks()
    # ---- the best single-step kernel of each automaton against the HBM roofline
    # (one step per launch: read and write every plane once), the word size
    # tuned for it as the workload leaves it open
    single = {}
    for a, g in grids.items():
        cells = torch.from_numpy(inputs.workload_grid(a, X, Y, SEED + rank)).to(dev)
        c1 = autotune.tune_word_bits(g["rule"], LAYOUT, cells, X, Y, word_bits=WORD_CHOICES[LAYOUT],
                                     candidates=autotune.SINGLE_STEP_CANDIDATES, use_cache=False)
        W1 = c1["word_bits"]
        if W1 == g["W"]:
            pa, pb = g["a"], g["b"]
            pa.buf.copy_(g["init"].buf)
        else:
            pa, pb = DevicePlanes(g["nb"], X, Y, dev), DevicePlanes(g["nb"], X, Y, dev)
            pa.pack_from(cells, LAYOUT, W1, sp)
        del cells
        n1 = 16
        autotune.run(c1, g["rule"], LAYOUT, W1, pa.ptrs, pb.ptrs, X, Y, 0, 2, sp)
        e0.record(stream)
        autotune.run(c1, g["rule"], LAYOUT, W1, pa.ptrs, pb.ptrs, X, Y, 0, n1, sp)
        e1.record(stream)
        torch.cuda.synchronize()
        ms1 = e0.elapsed_time(e1) / n1
        gbs = 2 * g["nb"] * g["init"].plane_bytes / (ms1 * 1e-3) / 1e9
        single[a] = {"kernel": describe_choice(c1), "word_bits": W1, "ms_per_step": round(ms1, 4),
                     "achieved_gbs": round(gbs, 1), "frac": round(gbs / peaks["hbm_gbs"], 4),
                     "gcups": round(X * Y / (ms1 * 1e-3) / 1e9, 1)}
        del pa, pb
        g["a"].buf.copy_(g["init"].buf)
    torch.cuda.synchronize()

    # ---- compute roofline of the temporal kernels: ALU-pipe instructions per
    # launch (ncu count of the configuration) over the live launch time, against
    # the ALU pipe's measured LOP3 rate on this device
    try:
        alu_peak = round(lop3_rate(sp) / 1e9, 1)
    except (OSError, RuntimeError, subprocess.CalledProcessError) as exc:  # the roofline is reported without it
        alu_peak, alu_err = None, repr(exc)[:200]
    alu = {"bound": "alu", "unit": "Gop/s (32-bit lane operations)", "peak": alu_peak,
           "peak_source": "measured live: lop3_rate.cu (independent lop3.b32 chains, full occupancy)"
           if alu_peak else f"unavailable: {alu_err}",
           "kernels": {}}
    # one capture per automaton: the timed configuration's when there is one
    picked = {}
    for key in MEASURED_ALU:
        a, lay, wb, k, th, loop, width, size = key
        if a not in grids or lay != LAYOUT or size != args.size or wb != grids[a]["W"]:
            continue
        c = {"mode": "temporal", "k": k, "tile_rows": th, "loop": loop, "width": width}
        timed = all(grids[a]["choice"].get(n) == v for n, v in c.items())
        if a not in picked or (timed and not picked[a][2]):
            picked[a] = (key, c, timed)
    for a, (key, c, timed) in picked.items():
        k = c["k"]
        count, src, fresh = measured(MEASURED_ALU, key, a)
        g = grids[a]
        nl = 8
        autotune.run(c, g["rule"], LAYOUT, g["W"], g["a"].ptrs, g["b"].ptrs, X, Y, 0, 2 * k, sp)
        e0.record(stream)
        autotune.run(c, g["rule"], LAYOUT, g["W"], g["a"].ptrs, g["b"].ptrs, X, Y, 0, nl * k, sp)
        e1.record(stream)
        torch.cuda.synchronize()
        msl = e0.elapsed_time(e1) / nl
        ach = count * 32 / (msl * 1e-3) / 1e9
        alu["kernels"][a] = {"kernel": describe_choice(c),
                             "timed_choice": timed,
                             "alu_warp_insts_per_launch": count, "ms_per_launch": round(msl, 4),
                             "achieved": round(ach, 1) if fresh else None,
                             "frac": round(ach / alu["peak"], 4) if fresh and alu["peak"] else None,
                             "alu_ops_per_cell_step": round(count * 32 / (X * Y * k), 2), "source": src,
                             "capture_matches_kernel_sources": fresh}
        g["a"].buf.copy_(g["init"].buf)
    torch.cuda.synchronize()

    # ---- roofline of the dominant kernel (the automaton with the most time)
    dom = max(AUTOMATA, key=lambda a: sum(per[a]))
    g = grids[dom]
    n_dom = launches(g) * diag_steps
    avg_launch_ms = sum(per[dom]) / n_dom
    bytes_per_launch = 2 * g["nb"] * g["init"].plane_bytes  # read + write every plane once per launch
    achieved = bytes_per_launch / (avg_launch_ms * 1e-3) / 1e9
    peak = peaks["hbm_gbs"]
    cap = measured(MEASURED_TRAFFIC, (dom, g["choice"]["mode"], g["choice"]["k"], args.size), dom)
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": cap[0] if cap and cap[2] else None,
            "traffic_source": (cap[1] if cap[2] else f"{cap[1]} (stale: captured from older kernel sources)")
            if cap else "no capture of this configuration",
            "kernel": f"{'temporal_kernel' if g['choice']['mode'] == 'temporal' else g['choice']['mode']} "
                      f"({dom}, k={g['choice']['k']})",
            "peak_source": peaks["source"],
            "bytes_per_launch": bytes_per_launch, "avg_launch_ms": round(avg_launch_ms, 4),
            # what the same GCUPS would need from HBM with one step per launch
            "single_step_equivalent_frac": round(per_gcups[dom] * 1e9 * g["nb"] / 4 / 1e9 / peak, 4)}

    if rank != 0:
        return None
    cpu = None
    if cpu_baseline and not args.no_cpu_baseline:
        kind, run = load_reference_cpu()
        th = host_threads()
        v, sample = cpu_sample(run, th, target_s=10.0)
        v1, sample1 = cpu_sample(run, 1, target_s=10.0)
        cpu = {"value": round(v, 4), "unit": "GCUPS", "cores": th, "kind": kind, "sample": sample,
               "single_core": {"value": round(v1, 4), "cores": 1, "sample": sample1}}
    line = {
        "metric": "GCUPS", "value": round(value, 1), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded i.i.d. grids)",
        "config": workload_config(args, extra={
            "traverser": {a: describe_choice(grids[a]["choice"]) for a in AUTOMATA},
            "parallelism": f"replicas x{world}",
            "automata_streams": "one after the other" if args.sequential else "one stream per automaton, concurrent"}),
        "per_automaton_note": "each automaton timed alone (2 steps) after the timed region",
        "per_automaton_gcups": {a: round(v, 1) for a, v in per_gcups.items()},
        "e2e": {"value": round(e2e_value, 1), "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "result_checked": bool(e2e_ok),
                "note": "pinned host planes through the C ABI; uploads and downloads on two copy streams, two "
                        "device plane sets per automaton used by alternate steps, so a step's copies overlap the "
                        "neighbouring steps' compute"},
        "gpu_launches": n_launch,
        "roofline": roof,
        "single_step_roofline": {"peak_gbs": peaks["hbm_gbs"], "peak_source": peaks["source"], **single},
        "alu_roofline": alu,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
    }
    return line


# ------------------------------------------------------- batched workload
def batched_arm(args, rank: int, world: int):
    """Many independent grids (mixed automata, log-uniform sides, aspect 1-4,
    uniform step counts) advanced by one CUDA-graph launch of the batch,
    against the same grids run one after another with per-grid launches."""
    import numpy as np
    import torch
    from cellato_b200 import inputs, lib
    from cellato_b200.batch import Batch
    from cellato_b200.device import DevicePlanes

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(SEED + rank)
    layout = LAYOUT
    specs = []
    lo, hi = np.log(args.batch_min_side), np.log(args.batch_max_side)
    for _ in range(args.batch_grids):
        rule = int(rng.integers(0, 10))
        side = float(np.exp(rng.uniform(lo, hi)))
        aspect = float(rng.uniform(1.0, 4.0))
        X, Y = side * np.sqrt(aspect), side / np.sqrt(aspect)
        if rng.integers(0, 2):
            X, Y = Y, X
        X = max(64, int(round(X / 64)) * 64)   # quantised: X a multiple of 64, Y of 16 (two 8-row tiles,
        Y = max(16, int(round(Y / 16)) * 16)   # even for critters), so that either word size fits
        steps = int(rng.integers(10, args.batch_max_steps + 1))
        specs.append((rule, X, Y, steps))
    gen = torch.Generator(device=dev)

    def cells_of(i):
        """Grid i's seeded initial state at its automaton's reference density."""
        rule, X, Y, _ = specs[i]
        probs = inputs.REFERENCE_DENSITY[inputs.RULES[rule]]
        vals = torch.tensor(list(probs.keys()), dtype=torch.uint8, device=dev)
        cum = torch.tensor(np.cumsum(list(probs.values())), dtype=torch.float64, device=dev)
        gen.manual_seed(SEED * 100003 + i)
        u = torch.rand((Y, X), generator=gen, device=dev, dtype=torch.float64)
        return vals[torch.clamp(torch.bucketize(u, cum), max=len(vals) - 1)].contiguous()

    # the autotuner: temporal depth per automaton on that automaton's median-sized
    # grid, at each word size; the batch takes the word size with the lower
    # total time over its cell updates (one word size holds for a whole batch)
    from cellato_b200 import autotune
    median = {}
    for r in sorted({s[0] for s in specs}):
        mine = sorted((X * Y, i) for i, (rr, X, Y, _) in enumerate(specs) if rr == r)
        median[r] = mine[len(mine) // 2][1]
    work = {r: sum(X * Y * s for rr, X, Y, s in specs if rr == r) for r in median}
    tuned = {}
    for W in WORD_CHOICES[layout]:
        for r, i in median.items():
            _, X, Y, _ = specs[i]
            sa, sb = DevicePlanes(inputs.PLANES[r], X, Y, dev), DevicePlanes(inputs.PLANES[r], X, Y, dev)
            sa.pack_from(cells_of(i), layout, W)
            tuned[(W, r)] = autotune.tune(r, layout, W, sa.ptrs, sb.ptrs, X, Y, candidates=BATCH_CANDIDATES,
                                          use_cache=False)
            del sa, sb
    W = min(WORD_CHOICES[layout], key=lambda w: sum(tuned[(w, r)]["ns_per_cell_step"] * work[r] for r in median))
    ks = {r: tuned[(W, r)]["k"] for r in median}

    bufs = []
    for i, (rule, X, Y, steps) in enumerate(specs):
        nb = inputs.PLANES[rule]
        a, b = DevicePlanes(nb, X, Y, dev), DevicePlanes(nb, X, Y, dev)
        a.pack_from(cells_of(i), layout, W)
        init = DevicePlanes(nb, X, Y, dev)
        init.buf.copy_(a.buf)
        bufs.append((a, b, init))
    torch.cuda.synchronize()
    cells_total = sum(X * Y * s for _, X, Y, s in specs)

    batch = Batch(layout, W, [(r, X, Y, s, a.ptrs, b.ptrs) for (r, X, Y, s), (a, b, _) in zip(specs, bufs)], ks)
    info = batch.info()
    sp = stream.cuda_stream
    for _ in range(args.warmup):
        batch.launch(sp)
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            batch.launch(sp)
        e1.record(stream)
        torch.cuda.synchronize()
    ms_batched = max_over_ranks(e0.elapsed_time(e1), world) / args.steps

    # results of one batched launch from the initial state, for the comparison
    for a, b, init in bufs:
        a.buf.copy_(init.buf)
    batch.launch(sp)
    torch.cuda.synchronize()
    batched_out = [((b if batch.result_in_b(i) else a).buf.clone()) for i, (a, b, _) in enumerate(bufs)]

    # plain per-grid launches of the same work
    for a, b, init in bufs:
        a.buf.copy_(init.buf)
    torch.cuda.synchronize()
    e0.record(stream)
    in_b = []
    for (rule, X, Y, s), (a, b, _) in zip(specs, bufs):
        in_b.append(lib.run_temporal(rule, layout, W, a.ptrs, b.ptrs, X, Y, 0, s, ks[rule], 0, sp))
    e1.record(stream)
    torch.cuda.synchronize()
    ms_per_grid = e0.elapsed_time(e1)
    mismatches = sum(0 if torch.equal(((b if f else a).buf), out) else 1
                     for (a, b, _), f, out in zip(bufs, in_b, batched_out))
    per_grid_launches = sum(-(-s // ks[r]) for r, _, _, s in specs)

    if rank != 0:
        return None
    value = cells_total * world / (ms_batched * 1e-3) / 1e9
    per_grid = cells_total / (ms_per_grid * 1e-3) / 1e9
    line = {
        "metric": "GCUPS", "value": round(value, 1), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_batched, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded, device-generated at reference densities)",
        "config": {"workload": f"batched: {args.batch_grids} grids, sides log-uniform {args.batch_min_side}-"
                               f"{args.batch_max_side}, aspect 1-4, 10 automata uniform, steps uniform "
                               f"10-{args.batch_max_steps}; tiled_bit_planes, word size and k autotuned; "
                               f"one CUDA-graph launch",
                   "k_per_automaton": {inputs.RULES[r]: k for r, k in ks.items()},
                   "word_bits": W,
                   "quantisation": "X to a multiple of 64, Y to a multiple of 16",
                   "cells_updates_per_step": cells_total, "graph_kernel_launches": info["kernel_launches"],
                   "work_items": info["work_items"]},
        "per_grid_launches_gcups": round(per_grid, 1),
        "batched_over_per_grid": round(value / world / per_grid, 2),
        "per_grid_kernel_launches": per_grid_launches,
        "bit_exact_vs_per_grid": mismatches == 0, "mismatching_grids": mismatches,
        "e2e": None, "e2e_note": "device-resident workload; see the config2 line for end-to-end",
        "gpu_launches": info["kernel_launches"] * args.steps,
        "clocks": clocks.summary(),
    }
    return line


def tune_temporal_k(dev, layout: int, W: int, sides) -> dict:
    """Temporal depth per automaton from the autotuner, measured on a scratch
    grid of each automaton at the given (X, Y)."""
    from cellato_b200 import autotune, inputs, lib
    from cellato_b200.device import DevicePlanes
    ks = {}
    for r, (X, Y) in sides.items():
        nb = inputs.PLANES[r]
        sa, sb = DevicePlanes(nb, X, Y, dev), DevicePlanes(nb, X, Y, dev)
        lib.fill_random(layout, W, nb, sa.ptrs, X, Y, SEED + r,
                        inputs.thresholds(inputs.REFERENCE_DENSITY[inputs.RULES[r]]))
        ks[r] = autotune.tune(r, layout, W, sa.ptrs, sb.ptrs, X, Y, candidates=BATCH_CANDIDATES,
                              use_cache=False)["k"]
        del sa, sb
    return ks


def served_arm(args, rank: int, world: int):
    """A Poisson stream of simulation requests through the continuous-batching
    server (cellato_server_*), then the same stream served one request at a time
    with plain per-grid launches.  Latency is measured from each request's
    scheduled arrival to the moment the host has its result (the 16 tile sums)."""
    import numpy as np
    import torch
    from cellato_b200 import inputs, lib
    from cellato_b200.device import DevicePlanes
    from cellato_b200.serve import Server

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    layout, W = LAYOUT, WORD_BITS
    rng = np.random.default_rng(SEED + 7 + rank)
    # arrivals over the window; sides and steps log-uniform; automata uniform
    t, arrivals = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / args.serve_rate))
        if t > args.serve_seconds:
            break
        arrivals.append(t)
    n = len(arrivals)
    reqs = []
    ls0, ls1 = np.log(args.serve_min_side), np.log(args.serve_max_side)
    lt0, lt1 = np.log(args.serve_min_steps), np.log(args.serve_max_steps)
    for i in range(n):
        r = int(rng.integers(0, 10))
        side = float(np.exp(rng.uniform(ls0, ls1)))
        X = max(64, int(round(side / 64)) * 64)
        Y = max(16, int(round(side / 16)) * 16)
        steps = int(round(np.exp(rng.uniform(lt0, lt1))))
        reqs.append((r, X, Y, steps, SEED * 1000003 + i))
    ths = {r: inputs.thresholds(inputs.REFERENCE_DENSITY[inputs.RULES[r]]) for r in range(10)}
    cell_updates = sum(X * Y * s for _, X, Y, s, _ in reqs)
    n_sample = min(n, max(3, int(round(n * args.serve_check_fraction))))
    sample = sorted(int(i) for i in rng.choice(n, size=n_sample, replace=False))
    ks = tune_temporal_k(dev, layout, W, {r: (1024, 1024) for r in range(10)})
    torch.cuda.synchronize()

    # ---- served; the plane pool may use 80% of the memory free now
    free_b, _ = torch.cuda.mem_get_info(dev)
    cap = int(0.8 * free_b)
    with ClockSampler(dev.index) as clocks:
        srv = Server(layout, W, hbm_cap_bytes=cap, k_per_rule=ks)
        lat, sums, ids = {}, {}, {}
        keep = set(sample)
        i = 0
        t0 = time.perf_counter()
        while len(lat) < n:
            now = time.perf_counter() - t0
            while i < n and arrivals[i] <= now:
                r, X, Y, steps, seed = reqs[i]
                ids[srv.submit_random(r, X, Y, steps, seed, thresholds=ths[r], keep=i in keep)] = i
                i += 1
            active = srv.iterate()
            for res in srv.poll():
                j = ids[res["id"]]
                lat[j] = time.perf_counter() - t0 - arrivals[j]
                sums[j] = res["checksum"]
            if active == 0 and srv.pending() == 0 and i < n:
                time.sleep(max(0.0, arrivals[i] - (time.perf_counter() - t0)))
        makespan = time.perf_counter() - t0
    stats = srv.stats()
    rid_of = {j: rid for rid, j in ids.items()}
    # the job: every rank's own stream, over the slowest rank's makespan
    job_cell_updates = sum_over_ranks(float(cell_updates), world)
    job_makespan = max_over_ranks(makespan * 1e3, world) / 1e3
    job_offered = int(sum_over_ranks(float(n), world))
    job_completed = int(sum_over_ranks(float(len(lat)), world))

    # ---- the sample: served planes against the same request run alone
    sample_ok = 0
    for j in sample:
        r, X, Y, steps, seed = reqs[j]
        nb = inputs.PLANES[r]
        a, b = DevicePlanes(nb, X, Y, dev), DevicePlanes(nb, X, Y, dev)
        lib.fill_random(layout, W, nb, a.ptrs, X, Y, seed, ths[r])
        in_b = lib.run_temporal(r, layout, W, a.ptrs, b.ptrs, X, Y, 0, steps, ks[r])
        alone = (b if in_b else a).download()
        served = lib.download_planes(nb, srv.planes(rid_of[j], nb), X * Y // 8)
        sample_ok += int(np.array_equal(alone, served))
        srv.release(rid_of[j])
        del a, b
    srv.close()

    # ---- the same stream, one request at a time with per-grid launches
    base = None
    if not args.no_per_grid:
        base_lat, mism = [], 0
        out = torch.zeros(16, dtype=torch.int64, device=dev)
        t0 = time.perf_counter()
        for j, (r, X, Y, steps, seed) in enumerate(reqs):
            wait = arrivals[j] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            nb = inputs.PLANES[r]
            a, b = DevicePlanes(nb, X, Y, dev), DevicePlanes(nb, X, Y, dev)
            lib.fill_random(layout, W, nb, a.ptrs, X, Y, seed, ths[r])
            in_b = lib.run_temporal(r, layout, W, a.ptrs, b.ptrs, X, Y, 0, steps, ks[r])
            lib.checksum(r, layout, W, (b if in_b else a).ptrs, X, Y, out.data_ptr())
            got = [int(v) & 0xFFFFFFFFFFFFFFFF for v in out.cpu().tolist()]
            base_lat.append(time.perf_counter() - t0 - arrivals[j])
            mism += int(got != sums[j])
        base_span = time.perf_counter() - t0
        job_base_span = max_over_ranks(base_span * 1e3, world) / 1e3
        base = {"gcups": round(job_cell_updates / job_base_span / 1e9, 1), "makespan_s": round(job_base_span, 3),
                "p50_ms": round(1e3 * float(np.percentile(base_lat, 50)), 1),
                "p99_ms": round(1e3 * float(np.percentile(base_lat, 99)), 1),
                "checksum_mismatches_vs_served": mism}

    if rank != 0:
        return None
    lats = np.array([lat[j] for j in range(n)])
    value = job_cell_updates / job_makespan / 1e9
    line = {
        "metric": "GCUPS", "value": round(value, 1), "unit": "GCUPS", "n_gpus": world, "steps": 1,
        "warmup": 0, "ms_per_step": round(job_makespan * 1e3, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded, device-generated at reference densities)",
        "config": {"workload": f"served: Poisson {args.serve_rate:g} req/s for {args.serve_seconds:g} s "
                               f"({n} requests), sides log-uniform {args.serve_min_side}-{args.serve_max_side}, "
                               f"steps log-uniform {args.serve_min_steps}-{args.serve_max_steps}, 10 automata "
                               f"uniform; tiled_bit_planes W64, k autotuned per automaton",
                   "k_per_automaton": {inputs.RULES[r]: k for r, k in ks.items()},
                   "quantisation": "X to a multiple of 64, Y to a multiple of 16",
                   "cell_updates": int(job_cell_updates),
                   "hbm_cap_bytes": cap,
                   "offered_gcups": round(job_cell_updates / args.serve_seconds / 1e9, 1),
                   "timing": "host wall clock from the first scheduled arrival to the last result"},
        "requests": {"offered": job_offered, "completed": job_completed,
                     "offered_gcups": round(job_cell_updates / args.serve_seconds / 1e9, 1),
                     "completed_gcups": round(value, 1),
                     "note": "every offered request completes; the offered load exceeds one GPU's rate, so the "
                             "queue and the latency grow with the arrival window"},
        "latency_ms": {"ranks": "rank 0's requests" if world > 1 else "all requests",
                       "p50": round(1e3 * float(np.percentile(lats, 50)), 1),
                       "p99": round(1e3 * float(np.percentile(lats, 99)), 1),
                       "max": round(1e3 * float(lats.max()), 1)},
        "per_grid": base,
        "served_over_per_grid": round(value / base["gcups"], 2) if base else None,
        "sample_bit_exact": f"{sample_ok}/{len(sample)}",
        "server": {"iterations": stats["iterations"], "kernel_launches": stats["kernel_launches"],
                   "pool_trims": stats["pool_trims"], "memory_waits": stats["memory_waits"],
                   "hbm_cap_bytes_at_end": stats["hbm_cap_bytes"]},
        "e2e": {"value": round(value, 1), "unit": "GCUPS", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": 128 * n,
                "note": "requests enter through the server's C ABI as seeds; results leave as 16 tile sums each"},
        "gpu_launches": stats["kernel_launches"],
        "clocks": clocks.summary(),
    }
    return line


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json)"}
    except (OSError, ValueError, KeyError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def sum_over_ranks(x: float, world: int) -> float:
    from cellato_b200 import replicas
    return replicas.sum_over_ranks(x) if world > 1 else x


def max_over_ranks(ms: float, world: int) -> float:
    from cellato_b200 import replicas
    return replicas.max_over_ranks(ms) if world > 1 else ms


def _free_device_memory():
    import gc
    import torch
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def _sub(line, keys):
    """The keys of a workload's own line kept beside the headline."""
    return {k: line[k] for k in keys if k in line}


def all_workloads(args, rank: int, world: int):
    """The config2 line with config3, batched and served beside it."""
    import copy
    apply_workload(args, "config2")
    line = our_arm(args, rank, world)
    _free_device_memory()
    a3 = copy.copy(args)
    a3.size = a3.ca_steps = None
    a3.choice = ""
    apply_workload(a3, "config3")
    c3 = our_arm(a3, rank, world, cpu_baseline=False)
    _free_device_memory()
    apply_workload(args, "config2")
    bt = batched_arm(args, rank, world)
    _free_device_memory()
    sv = served_arm(args, rank, world)
    _free_device_memory()
    if rank != 0:
        return
    line["config3"] = _sub(c3, ["value", "unit", "ms_per_step", "config", "per_automaton_gcups", "e2e",
                                "gpu_launches", "roofline", "single_step_roofline", "alu_roofline", "clocks"])
    line["batched"] = _sub(bt, ["value", "unit", "ms_per_step", "steps", "config", "per_grid_launches_gcups",
                                "batched_over_per_grid", "per_grid_kernel_launches", "bit_exact_vs_per_grid",
                                "mismatching_grids", "gpu_launches", "clocks"])
    line["served"] = _sub(sv, ["value", "unit", "config", "requests", "latency_ms", "per_grid",
                               "served_over_per_grid", "sample_bit_exact", "server", "e2e", "gpu_launches", "clocks"])
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    from cellato_b200 import replicas
    rank, world = replicas.init(timeout_s=120)
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world)
        elif args.workload == "all":
            all_workloads(args, rank, world)
        else:
            fn = {"batched": batched_arm, "served": served_arm}.get(args.workload, our_arm)
            line = fn(args, rank, world)
            if line is not None:
                print(json.dumps(line), flush=True)
    finally:
        replicas.shutdown()


if __name__ == "__main__":
    main()
