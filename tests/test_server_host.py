"""The native request loop's host logic on the CPU: mcv_sw_b200/csrc/mcv_server.cpp,
compiled unchanged with g++ against fake handle functions
(tests/native/fake_handles.cpp), run by tests/native/server_host_test.cpp.
Checks exact step counts and initial states per forecast, slot reuse, pools
per (order, Nc, dt), budget waits with eviction of idle empty pools, and that
no handle is touched while it has a chunk queued."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INC = "/usr/local/cuda/include"


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC), reason="needs g++ and CUDA headers")
def test_native_server_schedules_exactly(tmp_path):
    exe = tmp_path / "server_host_test"
    srcs = [os.path.join(ROOT, "mcv_sw_b200", "csrc", "mcv_server.cpp"),
            os.path.join(ROOT, "tests", "native", "fake_handles.cpp"),
            os.path.join(ROOT, "tests", "native", "server_host_test.cpp")]
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", CUDA_INC, *srcs, "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
