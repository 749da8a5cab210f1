"""The C++ front end (include/skgemm.hpp): a driver written against the
reference's class templates compiles and links against libskgemm.so alone
(CPU), and passes its known-answer checks on the GPU."""
import os
import subprocess

import pytest

import skgemm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "cpp", "reference_driver.cpp")


def _build(tmp_path):
    exe = str(tmp_path / "reference_driver")
    libdir = os.path.dirname(skgemm.LIB_PATH)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(REPO, "include"), SRC,
                    "-o", exe, "-L", libdir, "-lskgemm", f"-Wl,-rpath,{libdir}"],
                   check=True, capture_output=True, text=True)
    return exe


def test_driver_compiles_and_links(tmp_path):
    skgemm.lib()
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_driver_runs_on_gpu(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASSED" in r.stdout
