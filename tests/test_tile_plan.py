"""The register-tiled Bell kernels' plan, checked on the CPU by a small C++
program linked against the library's plan and table builders: the Horner
forward and the tiled correlation adjoint, run over the plan's records in
the kernels' loop order, reproduce the Bell recurrence and the pair sums
of every dense set with D0 <= 4 and K <= 7 (tests/cpp/tile_plan_check.cpp)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


def test_tile_plan_reproduces_the_bell_recurrence(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    csrc = os.path.join(ROOT, "dnnf90_b200", "csrc")
    exe = str(tmp_path / "tile_plan_check")
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", csrc,
                    os.path.join(ROOT, "tests", "cpp", "tile_plan_check.cpp"),
                    os.path.join(csrc, "tile_plan.cpp"), os.path.join(csrc, "tables.cpp"),
                    "-o", exe], check=True, timeout=300)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-3000:]
    assert "ALL OK" in out.stdout
    # the headline set: tiles over two dimensions, every slot covered
    assert "d0=4 k=7 na=330 ok=1 td=2" in out.stdout
