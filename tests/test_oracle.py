"""CPU: the oracle against the reference's own known answers.

Pins the oracle before anything is checked against it:
* the restated naive loops and the Dot2 oracle reproduce the golden vectors
  that the reference's own kernels produced on its own test inputs;
* where the reference kernels are built here (oracle/_ref), the restatements
  agree with them on further seeded shapes;
* Dot2 is checked against exact rational arithmetic on small cases.
"""
import ctypes
from fractions import Fraction

import numpy as np
import pytest

import oracle
from tests._cases import (GEMM_CASES, ROT_CASES, SYRK_CASES, gemm_inputs, golden_check,
                          rot_inputs, uniform)


@pytest.mark.parametrize("c", range(len(GEMM_CASES)))
def test_gemm_known_answers(golden, c):
    M, N, K, a, g = GEMM_CASES[c]
    A, B = gemm_inputs(M, N, K)
    D = oracle.gemm_naive(A, B, M, N, K, a, g)
    # The reference's tolerance is 1e-6 (gemm_opt.cpp:483); the oracle is far tighter.
    golden_check(golden, f"gemm{c}_opt", D, rtol=1e-13)
    golden_check(golden, f"gemm{c}_crsp", D, rtol=1e-13)
    Am = A.reshape(K, M).T
    Bm = B.reshape(K, N)
    D2 = oracle.dot2_matmul(Am, Bm, a, g)
    golden_check(golden, f"gemm{c}_opt", D2, rtol=1e-13)


@pytest.mark.parametrize("t", range(len(SYRK_CASES)))
def test_syrk_known_answers(golden, t):
    K, M = SYRK_CASES[t]
    Ap = oracle.init_A_packed_rand(K, M, 42 + t)
    assert np.allclose(golden[f"syrk{t}_A_checksum"], [Ap.sum(), (Ap * Ap).sum()], rtol=0, atol=0)
    C = oracle.syrk_naive(Ap, K, M, np.full(M * M, 0.1), 1.0, 0.0)
    Cm = C.reshape(M, M).T
    iu = np.triu_indices(M)
    golden_check(golden, f"syrk{t}_naive", Cm[iu], rtol=1e-13)
    golden_check(golden, f"syrk{t}_crsp", Cm[iu], rtol=1e-12)  # reference's tolerance: 1e-9
    A = oracle.unpack(Ap.reshape(-1, K, 16), M)  # (M, K)
    S = oracle.dot2_matmul(A, np.ascontiguousarray(A.T))
    golden_check(golden, f"syrk{t}_naive", S[iu], rtol=1e-13)


@pytest.mark.parametrize("t", range(len(ROT_CASES)))
def test_rot_known_answers(golden, t):
    Nd, nb = ROT_CASES[t]
    A, Q, Adense = rot_inputs(Nd, nb)
    D = oracle.rot_naive(A, Q, Nd, nb)
    golden_check(golden, f"rot{t}_naive", D, rtol=1e-13)
    golden_check(golden, f"rot{t}_sme", D, rtol=1e-12)  # reference's tolerance: 1e-9
    D2 = oracle.dot2_matmul(Adense, Q.reshape(nb, nb))
    golden_check(golden, f"rot{t}_naive", oracle.band_pack(D2).ravel(), rtol=1e-13)


def test_dot2_matches_exact_rationals():
    rng = np.random.default_rng(7)
    X = rng.standard_normal((5, 40)) * np.exp2(rng.integers(-30, 30, (5, 40)))
    Y = rng.standard_normal((40, 3)) * np.exp2(rng.integers(-30, 30, (40, 3)))
    got = oracle.dot2_matmul(X, Y, 1.5, 0.25)
    for i in range(5):
        for j in range(3):
            exact = sum(Fraction(X[i, k]) * Fraction(Y[k, j]) for k in range(40))
            exact = Fraction(1.5) * exact + Fraction(0.25)
            assert got[i, j] == float(exact) or abs(got[i, j] - float(exact)) <= 2 * abs(float(exact)) * 2**-53


def test_pack_roundtrip_and_c_pack():
    X = uniform((37, 11), 3)
    for T in (16, 32):
        P = oracle.pack(X, T)
        assert P.shape == ((37 + T - 1) // T, 11, T)
        assert np.array_equal(oracle.unpack(P, 37), X)
        Pc = np.zeros(P.size)
        oracle.lib().oracle_pack(37, 11, oracle.ptr(np.ascontiguousarray(X)), 11, 1, T,
                                 oracle.ptr(Pc))
        assert np.array_equal(Pc, P.ravel())
    Ab = oracle.band_pack(uniform((48, 32), 4))
    assert np.array_equal(oracle.band_unpack(Ab, 48), uniform((48, 32), 4))


# --------------------------------------------- the reference built in place
needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref not built")
_dp = ctypes.POINTER(ctypes.c_double)


@needs_ref
def test_reference_selftests_pass_under_emulation():
    """The reference's own known-answer drivers pass on the emulated intrinsics."""
    assert oracle.ref("gemm_opt").ref_gemm_opt_selftest() == 4
    assert oracle.ref("gemm_crsp").ref_gemm_crsp_selftest() == 4
    assert oracle.ref("syrk_crsp").ref_syrk_crsp_selftest() == 1
    assert oracle.ref("trp_3d").ref_trp_3d_selftest() == 6


@needs_ref
@pytest.mark.parametrize("M,N,K", [(48, 96, 300), (16, 32, 1), (128, 64, 777)])
def test_restatement_matches_reference_gemm(M, N, K):
    A = uniform(M * K, 10 + K)
    B = uniform(K * N, 20 + K)
    f = oracle.ref("gemm_opt").ref_gemm_opt_compute_test
    f.argtypes = [ctypes.c_int] * 3 + [_dp] * 3 + [ctypes.c_double] * 2
    D = np.zeros(M * N)
    f(M, N, K, oracle.ptr(A), oracle.ptr(B), oracle.ptr(D), 0.75, -0.125)
    ref = oracle.gemm_naive(A, B, M, N, K, 0.75, -0.125)
    assert oracle.rel_frobenius(D, ref) < 1e-14


@needs_ref
@pytest.mark.parametrize("K,M,alpha,beta", [(100, 48, 1.0, 0.0), (300, 64, 1.0, 0.5)])
def test_restatement_matches_reference_syrk(K, M, alpha, beta):
    Ap = oracle.pack(uniform((M, K), K), 16).ravel()
    C0 = uniform(M * M, 5)
    f = oracle.ref("sme_syrk").ref_sme_syrk_compute
    f.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double]
    C = C0.copy()
    f(K, M, oracle.ptr(Ap), oracle.ptr(C), alpha, beta)
    ref = oracle.syrk_naive(Ap, K, M, C0, alpha, beta)
    iu = np.triu_indices(M)
    assert oracle.rel_frobenius(C.reshape(M, M).T[iu], ref.reshape(M, M).T[iu]) < 1e-14


@needs_ref
def test_reference_quirks_documented():
    """Behaviours of the reference this library deliberately does not copy.

    Q2: gemm_opt drops the M%16 rows / N%32 columns (gemm_opt.cpp:318, :249).
    Q4: SYRK scales only the last 256-wide K chunk by alpha (sme_syrk.hpp:123-133).
    """
    M, N, K = 40, 40, 64
    A = uniform(M * K, 1)
    B = uniform(K * N, 2)
    f = oracle.ref("gemm_opt").ref_gemm_opt_compute_test
    f.argtypes = [ctypes.c_int] * 3 + [_dp] * 3 + [ctypes.c_double] * 2
    D = np.full(M * N, 7.0)
    f(M, N, K, oracle.ptr(A), oracle.ptr(B), oracle.ptr(D), 1.0, 0.0)
    D = D.reshape(M, N)
    assert np.all(D[32:, :] == 7.0) and np.all(D[:, 32:] == 7.0)  # never written
    K, M = 512, 32
    Ap = oracle.pack(uniform((M, K), 3), 16).ravel()
    g = oracle.ref("sme_syrk").ref_sme_syrk_compute
    g.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double]
    C = np.zeros(M * M)
    g(K, M, oracle.ptr(Ap), oracle.ptr(C), 2.0, 0.0)
    contract = oracle.syrk_naive(Ap, K, M, np.zeros(M * M), 2.0, 0.0)
    iu = np.triu_indices(M)
    assert oracle.rel_frobenius(C.reshape(M, M).T[iu], contract.reshape(M, M).T[iu]) > 0.1
