"""The serving loop's scheduling decisions on the CPU (polytope_b200/csrc/serve_sched.h, the code
server.cpp decides with): wave planning under the oldest-first and fair-share policies, admission
against the device-memory budget, and cancellation of queued requests and of admitted requests with
and without queued waves, in unit checks and in simulated scheduler runs (tests/cpp/serve_sched_check.cpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def test_serve_scheduling_decisions(tmp_path):
    exe = tmp_path / "serve_sched_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "polytope_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "serve_sched_check.cpp"), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == "ok", p.stdout + p.stderr
