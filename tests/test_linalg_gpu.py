"""The reference's C converter names (linalg_pack_c16_f64 / _r16 /
linalg_unpack_c16_f64 / _r16, include/sme_pack.hpp:316-352) exported by
libskgemm.so: bitwise against the oracle's grid packing, ragged Nd treated
as the reference does (only 16 * floor(Nd/16) grid points), and a plain C
caller that declares the reference's prototypes links and passes."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import skgemm

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("Nd,nb", [(4096, 512), (110592, 64), (1000, 48), (16, 1), (7, 32)])
def test_linalg_converters_bitwise(cuda, Nd, nb):
    R = Nd // 16 * 16
    X = np.random.default_rng(Nd + nb).standard_normal((Nd, nb))   # (g, b)
    colmajor = np.ascontiguousarray(X.T).ravel()                     # src[g + b*Nd]
    want = oracle.grid_pack(X[:R]).ravel()
    P = np.full(R * nb, np.nan)
    skgemm.sme_pack.pack_c16(Nd, nb, colmajor, P)
    assert np.array_equal(P, want)
    P2 = np.full(R * nb, np.nan)
    skgemm.sme_pack.pack_r16(Nd, nb, colmajor, P2)                 # row-major [nb, Nd]
    assert np.array_equal(P2, want)
    for name in ("unpack_c16", "unpack_r16"):
        Y = np.full(Nd * nb, -7.0)
        getattr(skgemm.sme_pack, name)(Nd, nb, want, Y)
        Y = Y.reshape(nb, Nd)
        assert np.array_equal(Y[:, :R], X[:R].T)
        assert np.all(Y[:, R:] == -7.0)   # rows past 16 * floor(Nd/16) untouched


def test_linalg_refusal_leaves_dst(cuda):
    P = np.full(16, 3.0)
    with pytest.raises(skgemm.SkgemmError):
        skgemm.sme_pack.pack_c16(-16, 1, np.zeros(16), P)
    assert np.all(P == 3.0)
    skgemm.sme_pack.pack_c16(16, 1, np.arange(16.0), P)   # a later call succeeds
    assert np.array_equal(P, np.arange(16.0))


def test_c_caller_with_reference_names(cuda, tmp_path):
    exe = str(tmp_path / "linalg_driver")
    libdir = os.path.dirname(skgemm.LIB_PATH)
    subprocess.run(["gcc", "-O2", os.path.join(REPO, "tests", "cpp", "linalg_driver.c"), "-o", exe,
                    "-L", libdir, "-lskgemm", f"-Wl,-rpath,{libdir}"],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "PASSED" in r.stdout, r.stdout + r.stderr
