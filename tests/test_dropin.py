"""The header-only C++ drop-in (include/fss_rhs_func.hpp) compiles against a
run_information-shaped struct and, on a GPU, runs the reference's call
pattern of rhs_func."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "fast-sphere-sum_b200", "fss_b200")


def build(tmp_path):
    exe = str(tmp_path / "dropin")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "dropin", "dropin_main.cpp"), "-L", LIBDIR, "-lfss",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_dropin_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_dropin_runs(tmp_path):
    out = subprocess.run([build(tmp_path)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "dropin ok" in out.stdout
