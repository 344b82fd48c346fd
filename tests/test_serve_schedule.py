"""The simulation server's scheduling policy (csrc/serve_schedule.hpp) compiled
for the host and driven through random request streams: FIFO admission under
the memory cap, the tile budget, and the per-request round sequence (buffers,
step parities, step counts) that makes a served result equal to a run alone."""
import os
import subprocess

from conftest import PKG, ROOT


def test_schedule_invariants(tmp_path):
    exe = str(tmp_path / "serve_schedule")
    subprocess.run(["g++", "-std=c++20", "-O1", "-Wall", f"-I{PKG}/csrc", "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "serve_schedule.cpp")], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
