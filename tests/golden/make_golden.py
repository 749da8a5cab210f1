"""Generates the golden vectors in this directory from the reference itself.

Runs the reference's own kernel files, compiled in place from the reference
tree by ``make -C oracle ref REF=<reference tree>`` (oracle/_ref), on the reference's own
known-answer inputs:

* gemm_opt.cpp / gemm_crsp.cpp test_gemm cases (M,N,K,alpha,gamma) =
  (32,64,128,1,0) (32,64,4096,1,0) (32,64,4096,2,.5) (64,128,2048,1,0) with the
  closed-form inputs of gemm_opt.cpp:444-453;
* syrk_crsp.cpp cases (K,M) = (64,32) (256,64) (512,96) (1024,128) (2048,256),
  seed 42+t through init_A_packed (syrk_crsp.cpp:379-395, host rand()),
  C preset to 0.1, alpha=1, beta=0 (syrk_crsp.cpp:474-505);
* trp_3d_test.cpp cases (Nd,nb) = (64,32) (256,64) (512,128) (1024,256)
  (2048,128) (4096,128) with the closed-form inputs of trp_3d_test.cpp:126-138.

Outputs are stored whole when small; larger ones as a fixed sample of
entries plus the sum and sum of squares of the whole output.

    python tests/golden/make_golden.py      (needs the reference tree)
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

import oracle  # noqa: E402

FULL_LIMIT = 16384
SAMPLE = 4096

GEMM_CASES = [(32, 64, 128, 1.0, 0.0), (32, 64, 4096, 1.0, 0.0), (32, 64, 4096, 2.0, 0.5),
              (64, 128, 2048, 1.0, 0.0)]
SYRK_CASES = [(64, 32), (256, 64), (512, 96), (1024, 128), (2048, 256)]
ROT_CASES = [(64, 32), (256, 64), (512, 128), (1024, 256), (2048, 128), (4096, 128)]


def gemm_inputs(M, N, K):
    """gemm_opt.cpp:444-453 closed-form inputs (A column-major, B row-major)."""
    i = np.arange(M)[:, None]
    j = np.arange(K)[None, :]
    A_col = np.ascontiguousarray(((i + 1) * 0.01 + (j + 1) * 0.001).T).ravel()  # A[i + j*M]
    k = np.arange(K)[:, None]
    n = np.arange(N)[None, :]
    B_row = ((k + 1) * 0.001 + (n + 1) * 0.01).ravel()
    return A_col, B_row


def rot_inputs(Nd, nb):
    """trp_3d_test.cpp:126-138: A(g,b) = (g+1)*0.001 + (b+1)*0.01 grid-packed,
    B[b*nb+bp] = (b+1)*0.01 + (bp+1)*0.001."""
    g = np.arange(Nd)[:, None]
    b = np.arange(nb)[None, :]
    A = (g + 1) * 0.001 + (b + 1) * 0.01
    bb = np.arange(nb)[:, None]
    bp = np.arange(nb)[None, :]
    Q = np.ascontiguousarray((bb + 1) * 0.01 + (bp + 1) * 0.001)
    return oracle.grid_pack(A).ravel(), Q.ravel(), A


def _store(out: dict, key: str, values: np.ndarray, seed: int):
    v = np.ascontiguousarray(values, dtype=np.float64).ravel()
    out[f"{key}_sum"] = np.array([v.sum()])
    out[f"{key}_sumsq"] = np.array([(v * v).sum()])
    out[f"{key}_size"] = np.array([v.size])
    if v.size <= FULL_LIMIT:
        out[f"{key}_idx"] = np.arange(v.size, dtype=np.int64)
    else:
        rng = np.random.default_rng(seed)
        out[f"{key}_idx"] = np.sort(rng.choice(v.size, SAMPLE, replace=False)).astype(np.int64)
    out[f"{key}_val"] = v[out[f"{key}_idx"]]


def main():
    dp = ctypes.POINTER(ctypes.c_double)
    P = oracle.ptr
    out = {}
    g_opt, g_crsp = oracle.ref("gemm_opt"), oracle.ref("gemm_crsp")
    for f in (g_opt.ref_gemm_opt_compute_test, g_crsp.ref_gemm_crsp_compute_test):
        f.argtypes = [ctypes.c_int] * 3 + [dp] * 3 + [ctypes.c_double] * 2
        f.restype = None
    for c, (M, N, K, a, gm) in enumerate(GEMM_CASES):
        A, B = gemm_inputs(M, N, K)
        for name, f in (("opt", g_opt.ref_gemm_opt_compute_test),
                        ("crsp", g_crsp.ref_gemm_crsp_compute_test)):
            D = np.zeros(M * N)
            f(M, N, K, P(A), P(B), P(D), a, gm)
            _store(out, f"gemm{c}_{name}", D, 100 + c)

    s_crsp = oracle.ref("syrk_crsp")
    s_crsp.ref_syrk_crsp_compute.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp,
                                             ctypes.c_double, ctypes.c_double]
    s_crsp.ref_syrk_crsp_reference.argtypes = s_crsp.ref_syrk_crsp_compute.argtypes
    s_crsp.ref_syrk_crsp_init_A_packed.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
    for t, (K, M) in enumerate(SYRK_CASES):
        Ap = np.zeros(((M + 15) // 16) * K * 16)
        s_crsp.ref_syrk_crsp_init_A_packed(K, M, P(Ap), 42 + t)
        out[f"syrk{t}_A_checksum"] = np.array([Ap.sum(), (Ap * Ap).sum()])
        for name, f in (("crsp", s_crsp.ref_syrk_crsp_compute),
                        ("naive", s_crsp.ref_syrk_crsp_reference)):
            C = np.full(M * M, 0.1)
            f(K, M, P(Ap), P(C), 1.0, 0.0)
            Cm = C.reshape(M, M).T  # column-major -> Cm[m1, m2] = C[m1 + m2*M]
            iu = np.triu_indices(M)
            _store(out, f"syrk{t}_{name}", Cm[iu], 200 + t)

    r = oracle.ref("trp_3d")
    r.ref_trp_3d_compute.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    r.ref_trp_3d_reference.argtypes = r.ref_trp_3d_compute.argtypes
    for t, (Nd, nb) in enumerate(ROT_CASES):
        A, Q, _ = rot_inputs(Nd, nb)
        for name, f in (("sme", r.ref_trp_3d_compute), ("naive", r.ref_trp_3d_reference)):
            D = np.zeros(Nd * nb)
            f(Nd, nb, P(A), P(Q), P(D))
            _store(out, f"rot{t}_{name}", D, 300 + t)

    path = os.path.join(HERE, "reference_known_answers.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
