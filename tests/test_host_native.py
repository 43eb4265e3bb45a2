"""Host-side native helpers of the transfer path, built on their own with
g++ and tested on the CPU:

* the worker pool of the transfer loops (sp3mm4amg_b200/csrc/host_pool.h):
  many short runs back to back, every index processed exactly once, no
  chunk running after its run returned;
* the cache of page-locked staging buffers (sp3mm4amg_b200/csrc/
  buffer_cache.h), with a fake allocator: its policy and 8 threads taking
  and giving buffers without sharing or leaking one."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "sp3mm4amg_b200", "csrc")

needs_gxx = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not found")


def _build(tmp_path, src):
    exe = str(tmp_path / os.path.splitext(src)[0])
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC,
                    os.path.join(HERE, src), "-o", exe], check=True)
    return exe


@needs_gxx
def test_host_pool_stress(tmp_path):
    exe = _build(tmp_path, "host_pool_stress.cpp")
    out = subprocess.run([exe, "100000", "7"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok"), out.stdout


@needs_gxx
def test_buffer_cache(tmp_path):
    exe = _build(tmp_path, "buffer_cache_test.cpp")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok"), out.stdout
