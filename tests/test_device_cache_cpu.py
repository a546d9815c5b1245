"""The per-device launch set-up memo (mdp_b200/csrc/device_cache.h), on the CPU.

cudaFuncSetAttribute applies to the current device only, so the library keys
each kernel's launch set-up by (kernel, shared-memory size, device).  This test
compiles tests/cpp/device_cache_test.cpp with g++ and runs it: set-up runs once
per key, a second device gets its own, failures are retried, and concurrent
first calls from 16 host threads run the set-up once per device.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_per_device_memo(tmp_path):
    exe = tmp_path / "device_cache_test"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-pthread", "-I", os.path.join(ROOT, "mdp_b200", "csrc"),
                           os.path.join(HERE, "cpp", "device_cache_test.cpp"), "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"
