"""The multi-GPU plumbing (replicas only: one process per GPU, no data-path
collective) run as two gloo ranks on the CPU: the barrier, the max over ranks
of the device time, the whole-job rate, and a two-rank launch of bench.py
through torch.distributed.run (its reference arm: rank 0 prints one line, the
other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import PKG, ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, queue):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, PKG)
    from cellato_b200 import replicas
    r, w = replicas.init(timeout_s=60, backend="gloo")
    replicas.barrier()
    slowest = replicas.max_over_ranks(10.0 + 5.0 * r)     # ms of this rank's timed region
    total = replicas.sum_over_ranks(1000.0 + r)            # work units that differ per rank
    queue.put((r, w, slowest, replicas.job_rate(2e9, w, slowest), total))
    replicas.barrier()
    replicas.shutdown()


def test_two_gloo_ranks_agree_on_the_slowest_time_and_the_sum():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[2] == 15.0 for o in out)              # both ranks see the max
    assert all(abs(o[3] - 2 * 2e9 / 15e-3) < 1 for o in out)
    assert all(o[4] == 2001.0 for o in out)            # both ranks see the sum


def test_bench_reference_arm_under_torchrun_two_ranks():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libcellato_ref.so")) and \
            not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        pytest.skip("oracle not built")
    env = dict(os.environ, PYTHONPATH=PKG)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, res.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
