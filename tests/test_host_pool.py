"""The host entry points' widening of 32-bit values into the caller's 64-bit
arrays and the thread pool that runs it (alpacc_b200/csrc/host_pool.h, host code
only), compiled with g++ and checked on the CPU by tests/host_pool_check.cpp."""

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_host_widening_pool(tmp_path):
    exe = str(tmp_path / "host_pool_check")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-pthread", "-o", exe,
                           os.path.join(HERE, "host_pool_check.cpp")])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
