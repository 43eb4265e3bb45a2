"""The host worker pool of the transfer loops (sp3mm4amg_b200/csrc/
host_pool.h), built on its own with g++ and stressed on the CPU: many short
runs back to back, every index processed exactly once, no chunk running
after its run returned."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "sp3mm4amg_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not found")
def test_host_pool_stress(tmp_path):
    exe = str(tmp_path / "host_pool_stress")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC,
                    os.path.join(HERE, "host_pool_stress.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe, "100000", "7"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok"), out.stdout
