"""CPU oracle — TEST INFRASTRUCTURE.

Used only by tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg, as the checker (never as the thing measured on the GPU, never shipped):

* ``liboracle.so`` (oracle.c): restatements of the reference's portable
  reference loops (gemm_opt.cpp:467-475, syrk_crsp.cpp:355-373,
  trp_3d_test.cpp:55-66) and a double-double (Dot2) accurate oracle;
* ``_ref/libref_*.so``: the reference's own kernel files compiled in place
  with a host emulation of the SME intrinsics they use (ref_shim/arm_sme.h),
  built by ``make ref`` where the reference tree exists and carried as built
  files elsewhere.

Parity status: pinned — the emulated reference passes all of its own
known-answer tests (gemm_opt 4/4, gemm_crsp 4/4, syrk_crsp 5/5, trp_3d 6/6),
and the restatements are checked against it in tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_f64p = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.c_int64
_lib: Optional[ctypes.CDLL] = None
_refs: dict = {}


def build(reference_root: Optional[str] = None) -> None:
    """make liboracle.so, and oracle/_ref from the reference source tree at
    `reference_root` (or $SKGEMM_REFERENCE_ROOT) when one is given and exists."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    reference_root = reference_root or os.environ.get("SKGEMM_REFERENCE_ROOT")
    if reference_root and os.path.isdir(reference_root):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={reference_root}"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_gemm_naive.argtypes = [_i64, _i64, _i64, _f64p, _f64p, _f64p,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.oracle_syrk_naive.argtypes = [_i64, _i64, _f64p, _f64p, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int]
        L.oracle_rot_naive.argtypes = [_i64, _i64, _f64p, _f64p, _f64p, ctypes.c_int]
        L.oracle_dot2_gemm.argtypes = [_i64, _i64, _i64, _f64p, _i64, _i64, _f64p, _i64, _i64,
                                       _f64p, _i64, _i64, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int]
        L.oracle_dot2_sampled.argtypes = [_i64, ctypes.POINTER(ctypes.c_int64),
                                          ctypes.POINTER(ctypes.c_int64), _i64, _f64p, _i64,
                                          _i64, _f64p, _i64, _i64, _f64p, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int]
        L.oracle_pack.argtypes = [_i64, _i64, _f64p, _i64, _i64, ctypes.c_int, _f64p]
        L.oracle_init_A_packed_rand.argtypes = [_i64, _i64, _f64p, ctypes.c_int]
        L.oracle_stencil_ext.argtypes = [_i64, _i64, _i64, _i64, ctypes.c_int, _f64p, _f64p,
                                         _f64p, _f64p, _f64p, ctypes.c_double, _f64p,
                                         ctypes.c_int, ctypes.c_int]
        L.oracle_halo_periodic.argtypes = [_i64, _i64, _i64, _i64, ctypes.c_int, _f64p, _f64p]
        _u32p = ctypes.POINTER(ctypes.c_uint32)
        _i32p = ctypes.POINTER(ctypes.c_int32)
        _i64p = ctypes.POINTER(ctypes.c_int64)
        L.oracle_nloc_project.argtypes = [_i64, _u32p, _u32p, _i32p, _u32p, _u32p, _i64p, _f64p,
                                          _i64p, _f64p, _i64p, _i64, _i64, ctypes.c_double,
                                          _f64p, _f64p, ctypes.c_int]
        for f in ("oracle_gemm_naive", "oracle_syrk_naive", "oracle_rot_naive",
                  "oracle_dot2_gemm", "oracle_dot2_sampled", "oracle_pack",
                  "oracle_init_A_packed_rand", "oracle_stencil_ext", "oracle_halo_periodic",
                  "oracle_nloc_project"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def naive_native() -> ctypes.CDLL:
    """The naive loops (oracle_gemm_naive / _syrk_naive / _rot_naive) built
    -O3 -march=native for this host (`make native`, built here on first use):
    the reference's portable kernels as a CPU baseline."""
    path = os.path.join(HERE, "_native", "liboracle_native.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", HERE, "native"], check=True)
    L = ctypes.CDLL(path)
    L.oracle_gemm_naive.argtypes = [_i64, _i64, _i64, _f64p, _f64p, _f64p,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int]
    L.oracle_syrk_naive.argtypes = [_i64, _i64, _f64p, _f64p, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int]
    L.oracle_rot_naive.argtypes = [_i64, _i64, _f64p, _f64p, _f64p, ctypes.c_int]
    for f in ("oracle_gemm_naive", "oracle_syrk_naive", "oracle_rot_naive"):
        getattr(L, f).restype = None
    return L


def ref(name: str) -> ctypes.CDLL:
    """The reference's own kernel file ``name`` built in place (oracle/_ref)."""
    if name not in _refs:
        path = os.path.join(REF_DIR, f"libref_{name}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref REF=<reference source tree>`")
        _refs[name] = ctypes.CDLL(path)
    return _refs[name]


def have_ref() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f"libref_{n}.so"))
               for n in ("gemm_opt", "gemm_crsp", "sme_syrk", "syrk_crsp", "trp_3d", "stencil",
                         "nloc"))


def ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_f64p)


def nthreads() -> int:
    return os.cpu_count() or 1


# ----------------------------------------------------------------- layouts
def pack(X: np.ndarray, T: int) -> np.ndarray:
    """(R, K) matrix -> packed-T panels [ceil(R/T)][K][T], zero padded."""
    R, K = X.shape
    tiles = (R + T - 1) // T
    P = np.zeros((tiles * T, K))
    P[:R] = X
    return np.ascontiguousarray(P.reshape(tiles, T, K).transpose(0, 2, 1))


def unpack(P: np.ndarray, R: int) -> np.ndarray:
    """packed-T panels [tiles][K][T] -> (R, K) matrix."""
    tiles, K, T = P.shape
    return np.ascontiguousarray(P.transpose(0, 2, 1).reshape(tiles * T, K)[:R])


def grid_pack(A: np.ndarray) -> np.ndarray:
    """(Nd, nb) states -> grid-packed [Nd/16][nb][16] (trp_3d_test.cpp:31-39)."""
    return pack(A, 16)


def band_pack(A: np.ndarray) -> np.ndarray:
    """(Nd, nb) states -> band-packed [nb/16][Nd][16] (trp_3d_test.cpp:41-49)."""
    return pack(np.ascontiguousarray(A.T), 16)


def band_unpack(P: np.ndarray, Nd: int) -> np.ndarray:
    tiles, Nd_, T = P.shape
    return np.ascontiguousarray(unpack(P, tiles * T).T[:Nd])


# ----------------------------------------------------------------- oracles
def gemm_naive(A_col: np.ndarray, B_row: np.ndarray, M, N, K, alpha=1.0, gamma=0.0,
               threads: int = 1) -> np.ndarray:
    D = np.zeros(M * N)
    lib().oracle_gemm_naive(M, N, K, ptr(A_col), ptr(B_row), ptr(D), alpha, gamma, threads)
    return D.reshape(M, N)


def syrk_naive(Ap: np.ndarray, K, M, C: np.ndarray, alpha=1.0, beta=0.0,
               threads: int = 1) -> np.ndarray:
    C = np.array(C, dtype=np.float64, order="C", copy=True)
    lib().oracle_syrk_naive(K, M, ptr(Ap), ptr(C), alpha, beta, threads)
    return C


def rot_naive(A_grid: np.ndarray, Q: np.ndarray, Nd, nb, threads: int = 1) -> np.ndarray:
    D = np.zeros(Nd * nb)
    lib().oracle_rot_naive(Nd, nb, ptr(A_grid), ptr(Q), ptr(D), threads)
    return D


def ext_size(ni, nj, nk, nb, FDn=6):
    """Doubles in an extended band-packed array [ceil(nb/16)][K_ex][16]."""
    return (nb + 15) // 16 * (ni + 2 * FDn) * (nj + 2 * FDn) * (nk + 2 * FDn) * 16


def stencil_ext(ext, A, ni, nj, nk, nb, cx, cy, cz, c0, out_tile=32, FDn=6, threads=1):
    """H Psi from extended band-packed Psi in the reference SVE kernels' order
    (stencil_extended_packed.hpp:47-181): [ceil(nb/T)][K][T] doubles."""
    K = ni * nj * nk
    out = np.zeros((nb + out_tile - 1) // out_tile * K * out_tile)
    lib().oracle_stencil_ext(ni, nj, nk, nb, FDn, ptr(ext), ptr(A), ptr(np.asarray(cx, float)),
                             ptr(np.asarray(cy, float)), ptr(np.asarray(cz, float)), c0,
                             ptr(out), out_tile, threads)
    return out


def stencil_naive(S_ex, A, ni, nj, nk, nb, cx, cy, cz, c0, FDn=6):
    """stencil_extended_test.cpp:200-236 restated with numpy: S_ex[b][k_ex][j_ex][i_ex]
    extended unpacked input, result [b][k][j][i]; x, then y, then z sums (not
    fused), the test's naive reference."""
    c = (slice(FDn, FDn + nk), slice(FDn, FDn + nj), slice(FDn, FDn + ni))
    res = S_ex[(slice(None),) + c] * (A.reshape(nk, nj, ni) + c0)
    for ax, coef in ((3, cx), (2, cy), (1, cz)):
        for r in range(1, FDn + 1):
            sp = [slice(None)] + list(c)
            sm = [slice(None)] + list(c)
            sp[ax] = slice(c[ax - 1].start + r, c[ax - 1].stop + r)
            sm[ax] = slice(c[ax - 1].start - r, c[ax - 1].stop - r)
            res = res + coef[r] * (S_ex[tuple(sp)] + S_ex[tuple(sm)])
    return res


def halo_periodic(local, ni, nj, nk, nb, FDn=6):
    """Single-rank periodic extension of band-packed Psi (halo_packed.hpp:93-124, :350-393)."""
    ext = np.zeros(ext_size(ni, nj, nk, nb, FDn))
    lib().oracle_halo_periodic(ni, nj, nk, nb, FDn, ptr(local), ptr(ext))
    return ext


class NlocProjectors:
    """A flattened nonlocal projector set: projector p has nrow[p] grid rows
    index[row_off[p]:], coefficients chi[chi_off[p]:] (column-major nrow x
    ncol), gamma[gam_off[p]:] (ncol), atom index atom[p] and its coefficient
    block at offsets[p] (offsets[P] = total columns) — the fields of the
    reference's Nloc_projector / Effective_potential_nloc."""

    def __init__(self, nrow, ncol, atom, offsets, index, chi, gamma):
        self.nrow = np.ascontiguousarray(nrow, dtype=np.uint32)
        self.ncol = np.ascontiguousarray(ncol, dtype=np.uint32)
        self.atom = np.ascontiguousarray(atom, dtype=np.int32)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        self.index = np.ascontiguousarray(index, dtype=np.uint32)
        self.chi = np.ascontiguousarray(chi, dtype=np.float64)
        self.gamma = np.ascontiguousarray(gamma, dtype=np.float64)
        P = len(self.nrow)
        self.row_off = np.concatenate([[0], np.cumsum(self.nrow.astype(np.int64))])[:P]
        self.chi_off = np.concatenate(
            [[0], np.cumsum(self.nrow.astype(np.int64) * self.ncol)])[:P].astype(np.int64)
        self.gam_off = np.concatenate([[0], np.cumsum(self.ncol.astype(np.int64))])[:P]
        self.row_off = np.ascontiguousarray(self.row_off, dtype=np.int64)
        self.gam_off = np.ascontiguousarray(self.gam_off, dtype=np.int64)

    def args(self):
        c = ctypes
        return (len(self.nrow), self.nrow.ctypes.data_as(c.POINTER(c.c_uint32)),
                self.ncol.ctypes.data_as(c.POINTER(c.c_uint32)),
                self.atom.ctypes.data_as(c.POINTER(c.c_int32)),
                self.offsets.ctypes.data_as(c.POINTER(c.c_uint32)),
                self.index.ctypes.data_as(c.POINTER(c.c_uint32)),
                self.row_off.ctypes.data_as(c.POINTER(c.c_int64)), ptr(self.chi),
                self.chi_off.ctypes.data_as(c.POINTER(c.c_int64)), ptr(self.gamma),
                self.gam_off.ctypes.data_as(c.POINTER(c.c_int64)))


def nloc_random(K, nrow, ncol, P, seed, images=1):
    """P atoms, each with `images` projectors that share its coefficient block
    (periodic images), unique grid rows per projector, chi ~ U[-1, 1), gamma ~
    0.5 U[-1, 1) (as nloc_packed_opt2_test.cpp:242-269 draws them)."""
    rng = np.random.default_rng(seed)
    nr, nc, at, off, idx, chi, gam = [], [], [], [], [], [], []
    col = 0
    for a in range(P):
        for _ in range(images):
            nr.append(nrow)
            nc.append(ncol)
            at.append(a + 1)
            off.append(col)
            idx.append(rng.permutation(K)[:nrow])
            chi.append(rng.uniform(-1, 1, nrow * ncol))
            gam.append(rng.uniform(-1, 1, ncol) * 0.5)
        col += ncol
    off.append(col)
    return NlocProjectors(nr, nc, at, off, np.concatenate(idx), np.concatenate(chi),
                          np.concatenate(gam))


def nloc_project(pj: NlocProjectors, psi16, nb, K, dv, out, out_tile=32):
    """out += V_nloc psi in the reference's order (oracle_nloc_project)."""
    lib().oracle_nloc_project(*pj.args(), nb, K, dv, ptr(psi16), ptr(out), out_tile)
    return out


def dot2_matmul(X: np.ndarray, Y: np.ndarray, alpha=1.0, gamma=0.0) -> np.ndarray:
    """alpha * X @ Y + gamma, every dot product in double-double (Dot2)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    M, K = X.shape
    K2, N = Y.shape
    assert K == K2
    out = np.zeros((M, N))
    lib().oracle_dot2_gemm(M, N, K, ptr(X), K, 1, ptr(Y), N, 1, ptr(out), N, 1, alpha, gamma,
                           nthreads())
    return out


def dot2_sampled(X: np.ndarray, Y: np.ndarray, ii: np.ndarray, jj: np.ndarray,
                 alpha=1.0, gamma=0.0, x_strides=None, y_strides=None, K=None) -> np.ndarray:
    """Entries (ii[t], jj[t]) of alpha * X @ Y + gamma in double-double.

    X is indexed X.flat[i*sxi + k*sxk] and Y Y.flat[k*syk + j*syj]; the default
    strides are those of C-contiguous (M, K) and (K, N) matrices."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    if K is None:
        K = X.shape[1]
    sxi, sxk = x_strides if x_strides else (X.shape[1], 1)
    syk, syj = y_strides if y_strides else (Y.shape[1], 1)
    ii = np.ascontiguousarray(ii, dtype=np.int64)
    jj = np.ascontiguousarray(jj, dtype=np.int64)
    out = np.zeros(len(ii))
    i64p = ctypes.POINTER(ctypes.c_int64)
    lib().oracle_dot2_sampled(len(ii), ii.ctypes.data_as(i64p), jj.ctypes.data_as(i64p), K,
                              ptr(X), sxi, sxk, ptr(Y), syk, syj, ptr(out), alpha, gamma,
                              nthreads())
    return out


def init_A_packed_rand(K: int, M: int, seed: int) -> np.ndarray:
    """syrk_crsp.cpp:379-395 seeded init (host C library rand())."""
    A = np.zeros(((M + 15) // 16) * K * 16)
    lib().oracle_init_A_packed_rand(K, M, ptr(A), seed)
    return A


def rel_frobenius(x: np.ndarray, ref: np.ndarray) -> float:
    ref = np.asarray(ref, dtype=np.float64).ravel()
    d = np.linalg.norm(np.asarray(x, dtype=np.float64).ravel() - ref)
    n = np.linalg.norm(ref.ravel())
    return float(d / n) if n > 0 else float(d)
