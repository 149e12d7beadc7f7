"""The tanh series forward's plan, checked on the CPU by a small C++
program linked against the library's plan and table builders."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


def test_series_plan_reproduces_the_bell_recurrence(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    csrc = os.path.join(ROOT, "dnnf90_b200", "csrc")
    exe = str(tmp_path / "series_plan_check")
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", csrc,
                    os.path.join(ROOT, "tests", "cpp", "series_plan_check.cpp"),
                    os.path.join(csrc, "bell_plan.cpp"), os.path.join(csrc, "tables.cpp"),
                    "-o", exe], check=True, timeout=300)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:]
    assert "ALL OK" in out.stdout
