"""Generates reference_hpsi.npz: golden outputs of the H Psi producers from the
reference itself. Uses the reference's own kernels, compiled in place from the
reference tree by ``make -C oracle ref REF=<reference tree>`` (oracle/_ref):

* calc_laplacian_extended_packed_16to32 / _16to16
  (include/stencil_extended_packed.hpp, through oracle/_ref/libref_stencil.so);
* Hamiltonian::nloc_project_vectors_packed / _16to16
  (include/nloc_packed_opt2.hpp, through oracle/_ref/libref_nloc.so).

The inputs are closed-form lattices of exactly representable values (integer
arithmetic scaled by powers of two), so every machine rebuilds them bit for bit
from the functions below; only the outputs are stored (whole when small, else
a fixed sample plus the sum and sum of squares, as make_golden.py does).

    python tests/golden/make_golden_hpsi.py      (needs the reference tree)
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

import oracle  # noqa: E402
from tests.golden.make_golden import _store  # noqa: E402

PATH = os.path.join(HERE, "reference_hpsi.npz")
FDN = 6
# 6th-order coefficients of stencil_extended_test.cpp:129-146 along x; y and z
# scaled by 1/2 and 1/4 (exact), so a swapped axis shows.
CX = [0.0, -1.0 / 12, 2.0 / 3, -2.5, 8.0 / 3, -1.0 / 4, 1.0 / 30]
CY = [c * 0.5 for c in CX]
CZ = [c * 0.25 for c in CX]
C0 = -0.5
STENCIL_CASES = [(7, 9, 6, 40), (8, 8, 8, 32), (5, 6, 13, 17)]  # (ni, nj, nk, nb)
# (K, nb, nrow, ncol, atoms, images, dv)
NLOC_CASES = [(600, 40, 50, 7, 3, 2, 0.03125), (900, 33, 120, 16, 4, 1, 0.0625)]


def lattice(n, a, b, m, scale):
    """((a i + b) mod m - m // 2) * scale for i < n: exact doubles."""
    i = np.arange(n, dtype=np.int64)
    return (((a * i + b) % m) - m // 2).astype(np.float64) * scale


def stencil_inputs(ni, nj, nk, nb):
    """Extended 16-band-packed Psi [tiles][Kx][16] (padding bands zero) and A."""
    kx = (ni + 2 * FDN) * (nj + 2 * FDN) * (nk + 2 * FDN)
    tiles = (nb + 15) // 16
    full = np.zeros((tiles * 16, kx))
    full[:nb] = lattice(nb * kx, 7919, 13, 2003, 2.0 ** -10).reshape(nb, kx)
    ext = np.ascontiguousarray(full.reshape(tiles, 16, kx).transpose(0, 2, 1)).ravel()
    A = lattice(ni * nj * nk, 31, 7, 101, 2.0 ** -4)
    return ext, A


def nloc_inputs(K, nb, nrow, ncol, atoms, images, T):
    """A projector set (periodic images share their atom's block), 16-band-
    packed psi and the T-packed output it is added to."""
    P = atoms * images
    nr, nc, at, off, idx = [], [], [], [], []
    col = 0
    for a in range(atoms):
        for m in range(images):
            p = a * images + m
            nr.append(nrow)
            nc.append(ncol)
            at.append(a + 1)
            off.append(col)
            idx.append((np.arange(nrow, dtype=np.int64) * 101 + 37 * p) % K)  # gcd(101, K) = 1
        col += ncol
    off.append(col)
    pj = oracle.NlocProjectors(nr, nc, at, off, np.concatenate(idx),
                               lattice(P * nrow * ncol, 13, 5, 257, 2.0 ** -8),
                               lattice(P * ncol, 29, 3, 61, 2.0 ** -6))
    psi16 = lattice((nb + 15) // 16 * K * 16, 7919, 11, 2003, 2.0 ** -10)
    base = lattice((nb + T - 1) // T * K * T, 613, 17, 1009, 2.0 ** -9)
    return pj, psi16, base


def main():
    out = {}
    st = oracle.ref("stencil")
    for c, (ni, nj, nk, nb) in enumerate(STENCIL_CASES):
        ext, A = stencil_inputs(ni, nj, nk, nb)
        K = ni * nj * nk
        for T, name in ((32, "ref_stencil_16to32"), (16, "ref_stencil_16to16")):
            o = np.zeros((nb + T - 1) // T * K * T)
            cx, cy, cz = (np.array(v, dtype=np.float64) for v in (CX, CY, CZ))
            getattr(st, name)(oracle.ptr(ext), oracle.ptr(o), oracle.ptr(A), ni, nj, nk, nb, FDN,
                              oracle.ptr(cx), oracle.ptr(cy), oracle.ptr(cz), ctypes.c_double(C0))
            mine = oracle.stencil_ext(ext, A, ni, nj, nk, nb, CX, CY, CZ, C0, T)
            assert np.array_equal(mine, o), (ni, nj, nk, nb, T)
            _store(out, f"stencil{c}_t{T}", o, 400 + 2 * c + T)
    nl = oracle.ref("nloc")
    cc = ctypes
    for c, (K, nb, nrow, ncol, atoms, images, dv) in enumerate(NLOC_CASES):
        for T in (32, 16):
            pj, psi16, base = nloc_inputs(K, nb, nrow, ncol, atoms, images, T)
            o = base.copy()
            a = pj.args()
            nl.ref_nloc_project(
                cc.c_int(a[0]), *a[1:6], pj.row_off.ctypes.data_as(cc.POINTER(cc.c_longlong)),
                a[7], pj.chi_off.ctypes.data_as(cc.POINTER(cc.c_longlong)), a[9],
                pj.gam_off.ctypes.data_as(cc.POINTER(cc.c_longlong)), cc.c_int(nb), cc.c_int(K),
                cc.c_double(dv), oracle.ptr(psi16), oracle.ptr(o), cc.c_int(T))
            mine = oracle.nloc_project(pj, psi16, nb, K, dv, base.copy(), T)
            assert np.array_equal(mine, o), (K, nb, T)
            assert not np.array_equal(o, base)
            _store(out, f"nloc{c}_t{T}", o, 500 + 2 * c + T)
    np.savez_compressed(PATH, **out)
    print(PATH, os.path.getsize(PATH), "bytes")


if __name__ == "__main__":
    main()
