"""The C++ front end (include/skgemm.hpp): a driver written against the
reference's class templates compiles and links against libskgemm.so alone
(CPU), and passes its known-answer checks on the GPU."""
import os
import subprocess

import pytest

import skgemm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "cpp", "reference_driver.cpp")


def _build(tmp_path, src=SRC):
    exe = str(tmp_path / os.path.splitext(os.path.basename(src))[0])
    libdir = os.path.dirname(skgemm.LIB_PATH)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(REPO, "include"), src,
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


def test_sme_pack_host_converters(tmp_path):
    """sme_pack<double> (host loops, no GPU) against the layouts' index maps."""
    skgemm.lib()
    exe = _build(tmp_path, os.path.join(REPO, "tests", "cpp", "pack_driver.cpp"))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "PASSED" in r.stdout, r.stdout + r.stderr
