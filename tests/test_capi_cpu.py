"""CPU: the C ABI library loads, exports every entry point include/skgemm.h
declares, and rejects bad arguments before touching a device. No compute
call is made here (there is no GPU on the CPU runner)."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import skgemm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(name="skgemm.h"):
    src = open(os.path.join(REPO, "include", name)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(skgemm_[a-z0-9_]+)\s*\(", src)))


def test_library_builds_and_loads():
    L = skgemm.lib()
    assert skgemm.version().startswith("skgemm")
    assert isinstance(L, ctypes.CDLL)


def test_every_declared_symbol_is_exported():
    declared = header_functions()
    assert len(declared) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", skgemm.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (skgemm_[a-z0-9_]+)", out))
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    # and the binding knows every one of them
    assert set(declared) <= set(skgemm.exported_symbols())


def test_only_the_abi_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", skgemm.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    text_syms = re.findall(r"\bT (\S+)", out)
    assert all(s.startswith("skgemm_") or s in skgemm.LINALG for s in text_syms), text_syms


def test_reference_converter_names_exported():
    """The reference's own extern "C" names (include/sme_pack.hpp:316-352) are
    declared in the header with the reference's signature and exported, so a
    caller linked against them resolves."""
    src = open(os.path.join(REPO, "include", "skgemm.h")).read()
    out = subprocess.run(["nm", "-D", "--defined-only", skgemm.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    for name in skgemm.LINALG:
        assert re.search(rf"\bvoid {name}\(const int Nd, const int nb, const double\* src, "
                         rf"double\* dst\);", src), name
        assert re.search(rf"\bT {name}\b", out), name


@pytest.mark.parametrize("call", [
    lambda: skgemm.gemm.compute_test(-1, 4, 4, np.zeros(16), np.zeros(16), np.zeros(16)),
    lambda: skgemm.gemm.compute_packed(4, -4, 4, np.zeros(16), np.zeros(16), np.zeros(16)),
    lambda: skgemm.sme_syrk.compute(-3, 4, np.zeros(64), np.zeros(16)),
    lambda: skgemm.sme_gemm_trp_3d.compute(20, 16, np.zeros(320), np.zeros(256), np.zeros(320)),
    lambda: skgemm.sme_gemm_trp_3d.compute(16, -16, np.zeros(1), np.zeros(1), np.zeros(1)),
])
def test_invalid_arguments_rejected_without_device(call):
    with pytest.raises(skgemm.SkgemmError) as e:
        call()
    assert e.value.code == skgemm.ERR_INVALID_ARG


def test_host_arrays_must_be_float64_contiguous():
    with pytest.raises(skgemm.SkgemmError):
        skgemm.gemm.compute_test(2, 2, 2, np.zeros(4, dtype=np.float32), np.zeros(4),
                                 np.zeros(4))
    with pytest.raises(skgemm.SkgemmError):
        skgemm.gemm.compute_test(2, 2, 2, np.zeros((4, 2))[:, 0], np.zeros(4), np.zeros(4))


def test_no_silent_cpu_fallback():
    """A well-formed call without an sm_100 device fails loudly."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.gemm.compute_test(2, 2, 2, np.ones(4), np.ones(4), np.zeros(4))
    assert e.value.code in (skgemm.ERR_NO_DEVICE, skgemm.ERR_CUDA)


def test_debug_fill_switch_read_from_environment():
    """SKGEMM_DEBUG_FILL=1 turns the debug fill mode on for the process
    (read once); it is off otherwise. No device is needed to ask."""
    assert skgemm.debug_fill() is False
    code = ("import sys; sys.path.insert(0, %r); import skgemm; "
            "print(int(skgemm.debug_fill()))" % os.path.join(REPO, "stream-k-gemm_b200"))
    for val, want in (("1", "1"), ("0", "0")):
        env = dict(os.environ, SKGEMM_DEBUG_FILL=val)
        out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True,
                             text=True, check=True).stdout.strip()
        assert out == want, (val, out)
