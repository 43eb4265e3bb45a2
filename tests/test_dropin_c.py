"""The drop-in boundary from C: a C11 program (tests/dropin_driver.c) that
includes include/sp3mm_b200.h, links lib/libsp3mm_b200.so and walks the
reference's dispatch tables as the reference's test driver does
(code/test/Sp3MM_test.c:355-419), freeing every result with free().

On the CPU the driver is compiled and linked (the header and the exported
symbols serve a C caller); on the GPU it runs on golden cases in both index
bases and every result must equal the reference's, bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = str(tmp_path / "dropin_driver")
    subprocess.run(["gcc", "-std=c11", "-O1", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "dropin_driver.c"),
                    "-o", exe, capi.LIB_PATH, "-Wl,-rpath," + os.path.dirname(capi.LIB_PATH)],
                   check=True)
    return exe


def test_c_driver_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
@pytest.mark.parametrize("off", [0, 1])
def test_c_driver_walks_dispatch_tables(golden, tmp_path, off):
    exe = _build(tmp_path)
    for name in ("poisson2d_64_agg2", "random_rect_empty_rows"):
        g = golden[name]
        d = tmp_path / f"{name}_{off}"
        d.mkdir()
        paths = []
        for k in ("R", "A", "P"):
            p = str(d / f"{k}.mtx")
            S.write_mm(g[k], p)
            paths.append(p)
        out = subprocess.run([exe, *paths, str(d), str(off)], capture_output=True, text=True)
        assert out.returncode == 0, out.stderr
        n = int(out.stdout.strip())
        # 4 UB pair-wise + 1 UB direct, then 2 x (2 SymbNum pair-wise + 1 direct).
        assert n == 4 + 1 + 2 * (2 + 1)
        files = sorted(f for f in os.listdir(d) if f.endswith(".mtx") and f[0] in "pd")
        assert len(files) == n
        for f in files:
            got = S.read_mm(str(d / f), sort_rows=False)
            want = g["direct"] if f.startswith("direct") else g["pair"]
            cmp = O.compare(got, want, rtol=0.0)
            assert cmp["ok"] and cmp["bitwise_equal"] == want.nnz, (name, off, f, cmp)
