"""GPU parity of the native FP64 Stream-K path, called through the C ABI.

Gates:
* the reference's own known-answer cases reproduce the golden vectors its
  kernels produced (scaled error <= 1e-12; the reference's tolerance is 1e-6
  for GEMM, 1e-9 for SYRK and the rotation);
* every other case: relative Frobenius error <= 1e-13 against the Dot2
  (double-double) oracle;
* full-size configurations are checked on a sample of entries against Dot2
  plus size-independent properties.
"""
import numpy as np
import pytest
import torch

import oracle
import skgemm
from tests._cases import (GEMM_CASES, ROT_CASES, SYRK_CASES, gaussian, gemm_inputs,
                          golden_check, rot_inputs, uniform)

pytestmark = pytest.mark.gpu
TOL = 1e-13  # relative Frobenius error vs the Dot2 oracle


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ------------------------------------------------------------------ GEMM
@pytest.mark.parametrize("c", range(len(GEMM_CASES)))
def test_gemm_known_answers_host_api(cuda, golden, c):
    M, N, K, a, g = GEMM_CASES[c]
    A, B = gemm_inputs(M, N, K)
    D = np.zeros(M * N)
    skgemm.gemm.compute_test(M, N, K, A, B, D, a, g)
    golden_check(golden, f"gemm{c}_opt", D, rtol=1e-12)
    ref = oracle.dot2_matmul(A.reshape(K, M).T, B.reshape(K, N), a, g)
    assert oracle.rel_frobenius(D, ref) <= TOL
    # Same case through the packed entry point (gemm_opt.cpp:314 / gemm_crsp.cpp:316).
    Ap = oracle.pack(A.reshape(K, M).T, 16).ravel()
    Bp = oracle.pack(B.reshape(K, N).T, 32).ravel()
    D2 = np.zeros(M * N)
    skgemm.gemm.compute_streamk_packed(M, N, K, Ap, Bp, D2, a, g)
    golden_check(golden, f"gemm{c}_crsp", D2, rtol=1e-12)


def test_gemm_config1_1000_rowmajor(cuda):
    """M=N=K=1000 (not a tile multiple), row-major A and B, U[-1,1] entries."""
    M = N = K = 1000
    A = uniform((M, K), 2024)
    B = uniform((K, N), 2025)
    dA, dB = dev(A), dev(B)
    Ap = torch.empty(((M + 15) // 16) * 16 * K, dtype=torch.float64, device="cuda")
    Bp = torch.empty(((N + 31) // 32) * 32 * K, dtype=torch.float64, device="cuda")
    skgemm.pack_dev(M, K, dA, K, 1, 16, Ap)   # A(m, k) = A[m*K + k]
    skgemm.pack_dev(N, K, dB, 1, N, 32, Bp)   # B(n, k) = B[k*N + n]
    dD = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
    skgemm.dgemm_packed_dev(M, N, K, Ap, Bp, dD)
    skgemm.stream_status()
    D = host(dD)
    ref = oracle.dot2_matmul(A, B)
    err = oracle.rel_frobenius(D, ref)
    assert err <= TOL, err
    naive = oracle.gemm_naive(np.ascontiguousarray(A.T).ravel(), B.ravel(), M, N, K,
                              threads=oracle.nthreads())
    assert oracle.rel_frobenius(D, naive) <= TOL


@pytest.mark.parametrize("M,N,K,a,g", [
    (1, 1, 1, 1.0, 0.0), (7, 13, 5, 2.0, 0.5), (17, 33, 100, -1.5, 3.0),
    (129, 65, 257, 1.0, 0.0), (200, 300, 1000, 0.5, -0.25), (16, 32, 16, 1.0, 1.0),
    (333, 129, 4099, 1.0, 0.0), (1, 515, 31, 1.0, 0.0), (515, 1, 33, 1.0, 0.0)])
def test_gemm_shapes_dense_and_packed(cuda, M, N, K, a, g):
    A = uniform((M, K), M * 7 + K)
    B = uniform((K, N), N * 5 + K)
    ref = oracle.dot2_matmul(A, B, a, g)
    # dense: A column-major (lda = M), B row-major (ldb = N)
    dA = dev(np.ascontiguousarray(A.T))
    dB = dev(B)
    dD = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
    skgemm.dgemm_dev(M, N, K, dA, M, dB, N, dD, N, a, g)
    skgemm.stream_status()
    assert oracle.rel_frobenius(host(dD), ref) <= TOL
    # packed
    Ap, Bp = dev(oracle.pack(A, 16)), dev(oracle.pack(np.ascontiguousarray(B.T), 32))
    dD2 = torch.full((M, N + 3), np.nan, dtype=torch.float64, device="cuda")
    skgemm.dgemm_packed_dev(M, N, K, Ap, Bp, dD2, N + 3, a, g)
    skgemm.stream_status()
    D2 = host(dD2)
    assert oracle.rel_frobenius(D2[:, :N], ref) <= TOL
    assert np.all(np.isnan(D2[:, N:]))  # padding columns untouched


def test_gemm_odd_leading_dimension_packs_first(cuda):
    M, N, K = 37, 41, 300
    A = uniform((M, K), 1)
    B = uniform((K, N), 2)
    lda, ldb = M + 1, N  # ldb = 41 is odd: packed on the device first
    Acol = np.zeros((K, lda))
    Acol[:, :M] = A.T
    dD = torch.zeros((M, N), dtype=torch.float64, device="cuda")
    skgemm.dgemm_dev(M, N, K, dev(Acol), lda, dev(B), ldb, dD, N, 1.0, 0.0)
    skgemm.stream_status()
    assert oracle.rel_frobenius(host(dD), oracle.dot2_matmul(A, B)) <= TOL


def test_gemm_k_zero_and_empty(cuda):
    dD = torch.zeros((5, 6), dtype=torch.float64, device="cuda")
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    skgemm.dgemm_packed_dev(5, 6, 0, dummy, dummy, dD, 6, 2.0, 0.75)
    skgemm.stream_status()
    assert np.all(host(dD) == 0.75)
    skgemm.dgemm_packed_dev(0, 6, 10, dummy, dummy, dD, 6, 1.0, 0.0)  # no-op
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.dgemm_packed_dev(-1, 6, 10, dummy, dummy, dD, 6)
    assert e.value.code == skgemm.ERR_INVALID_ARG


def test_gemm_deterministic_streamk(cuda):
    """Stream-K fixup order is fixed: two runs are bitwise identical."""
    M, N, K = 512, 512, 65536  # 16 tiles, each split over ~9 CTAs
    A = gaussian((M, K), 5)
    B = gaussian((K, N), 6)
    Ap, Bp = dev(oracle.pack(A, 16)), dev(oracle.pack(np.ascontiguousarray(B.T), 32))
    outs = []
    for _ in range(2):
        dD = torch.zeros((M, N), dtype=torch.float64, device="cuda")
        skgemm.dgemm_packed_dev(M, N, K, Ap, Bp, dD)
        skgemm.stream_status()
        outs.append(host(dD))
    assert np.array_equal(outs[0], outs[1])
    ii = np.random.default_rng(0).integers(0, M, 256)
    jj = np.random.default_rng(1).integers(0, N, 256)
    ref = oracle.dot2_sampled(A, B, ii, jj)
    assert oracle.rel_frobenius(outs[0][ii, jj], ref) <= TOL


# ------------------------------------------------------------------ SYRK
@pytest.mark.parametrize("t", range(len(SYRK_CASES)))
def test_syrk_known_answers_host_api(cuda, golden, t):
    K, M = SYRK_CASES[t]
    Ap = oracle.init_A_packed_rand(K, M, 42 + t)
    C = np.full(M * M, 0.1)
    skgemm.sme_syrk.compute(K, M, Ap, C, 1.0, 0.0)
    Cm = C.reshape(M, M).T
    iu = np.triu_indices(M)
    golden_check(golden, f"syrk{t}_naive", Cm[iu], rtol=1e-12)
    golden_check(golden, f"syrk{t}_crsp", Cm[iu], rtol=1e-12)
    il = np.tril_indices(M, -1)
    assert np.all(Cm[il] == 0.1)  # strict lower triangle untouched


@pytest.mark.parametrize("K,M,alpha,beta", [
    (1, 1, 1.0, 0.0), (77, 5, 1.7, 0.0), (1000, 16, 1.0, -0.3), (300, 100, -0.5, 2.0),
    (4096, 130, 1.0, 0.0), (513, 257, 3.0, 0.5), (20000, 512, 1.0, 0.0)])
def test_syrk_shapes(cuda, K, M, alpha, beta):
    A = uniform((M, K), K + M)
    Ap = oracle.pack(A, 16).ravel()
    C0 = uniform(M * M, 9)
    C = C0.copy()
    skgemm.sme_syrk.compute(K, M, Ap, C, alpha, beta)
    Cm = C.reshape(M, M).T
    C0m = C0.reshape(M, M).T
    ref = oracle.dot2_matmul(A, np.ascontiguousarray(A.T), alpha) + beta * C0m
    iu = np.triu_indices(M)
    assert oracle.rel_frobenius(Cm[iu], ref[iu]) <= TOL
    il = np.tril_indices(M, -1)
    assert np.array_equal(Cm[il], C0m[il])


def test_syrk_device_ldc_and_nan_beta_zero(cuda):
    """beta == 0 must not read C (NaN in C does not propagate), as in the
    reference's store path (sme_syrk.hpp:73-75)."""
    K, M, ldc = 700, 70, 75
    A = uniform((M, K), 3)
    dC = torch.full((M, ldc), np.nan, dtype=torch.float64, device="cuda")  # column j = row j
    skgemm.dsyrk_packed_dev(K, M, dev(oracle.pack(A, 16)), dC, ldc, 2.0, 0.0)
    skgemm.stream_status()
    C = host(dC)[:, :M].T  # C[m1, m2] = buf[m2*ldc + m1]
    ref = oracle.dot2_matmul(A, np.ascontiguousarray(A.T), 2.0)
    iu = np.triu_indices(M)
    assert oracle.rel_frobenius(C[iu], ref[iu]) <= TOL


# -------------------------------------------------------------- rotation
@pytest.mark.parametrize("t", range(len(ROT_CASES)))
def test_rot_known_answers_host_api(cuda, golden, t):
    Nd, nb = ROT_CASES[t]
    A, Q, Adense = rot_inputs(Nd, nb)
    D = np.zeros(Nd * nb)
    skgemm.sme_gemm_trp_3d.compute(Nd, nb, A, Q, D)
    golden_check(golden, f"rot{t}_sme", D, rtol=1e-12)
    golden_check(golden, f"rot{t}_naive", D, rtol=1e-12)
    ref = oracle.band_pack(oracle.dot2_matmul(Adense, Q.reshape(nb, nb))).ravel()
    assert oracle.rel_frobenius(D, ref) <= TOL


@pytest.mark.parametrize("Nd,nb", [(16, 16), (48, 80), (1024, 528), (4096, 1024)])
def test_rot_shapes(cuda, Nd, nb):
    Psi = gaussian((Nd, nb), Nd + nb, 1 / np.sqrt(Nd))
    Q = uniform((nb, nb), 11)
    dD = torch.full((Nd * nb,), np.nan, dtype=torch.float64, device="cuda")
    skgemm.drot_dev(Nd, nb, dev(oracle.grid_pack(Psi)), dev(Q), dD)
    skgemm.stream_status()
    ref = oracle.band_pack(oracle.dot2_matmul(Psi, Q)).ravel()
    assert oracle.rel_frobenius(host(dD), ref) <= TOL


@pytest.mark.parametrize("Nd,nb", [(16, 16), (48, 80), (1024, 528), (4096, 512), (2000, 400),
                                   (20000, 512), (4096, 1024)])
def test_rot_band_equals_grid(cuda, Nd, nb):
    """skgemm_drot_band_dev on band-packed Psi (the transposition folded into
    the K-major loads) equals skgemm_drot_dev on the grid-packed copy, bit for
    bit (same tiles, schedule and k order), and Dot2 within the gate. The
    shapes cover both tile kernels (128 x 128 for few tiles, 64 x 64)."""
    Psi = gaussian((Nd, nb), Nd + 3 * nb, 1 / np.sqrt(Nd))
    Q = dev(uniform((nb, nb), 12))
    grid = torch.full((Nd * nb,), np.nan, dtype=torch.float64, device="cuda")
    band = torch.full((Nd * nb,), np.nan, dtype=torch.float64, device="cuda")
    skgemm.drot_dev(Nd, nb, dev(oracle.grid_pack(Psi)), Q, grid)
    skgemm.drot_band_dev(Nd, nb, dev(oracle.band_pack(Psi)), Q, band)
    skgemm.stream_status()
    assert torch.equal(band, grid)
    ref = oracle.band_pack(oracle.dot2_matmul(Psi, host(Q).reshape(nb, nb))).ravel()
    assert oracle.rel_frobenius(host(band), ref) <= TOL


def test_rot_band_rejects_ragged(cuda):
    A = torch.zeros(48 * 40, dtype=torch.float64, device="cuda")
    q = torch.zeros(40 * 40, dtype=torch.float64, device="cuda")
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.drot_band_dev(48, 40, A, q, torch.zeros_like(A))
    assert e.value.code == skgemm.ERR_INVALID_ARG


# --------------------------------------------------------- layout kernels
def test_band_grid_roundtrip_device(cuda):
    Nd, nb = 272, 96
    Psi = gaussian((Nd, nb), 1)
    band = dev(oracle.band_pack(Psi))
    grid = torch.zeros(Nd * nb, dtype=torch.float64, device="cuda")
    skgemm.band_to_grid_dev(Nd, nb, band, grid)
    assert np.array_equal(host(grid), oracle.grid_pack(Psi).ravel())
    back = torch.zeros(Nd * nb, dtype=torch.float64, device="cuda")
    skgemm.grid_to_band_dev(Nd, nb, grid, back)
    assert np.array_equal(host(back), host(band).ravel())


def test_pack_device_matches_oracle(cuda):
    R, K = 45, 70
    X = uniform((R, K), 8)
    for T in (16, 32):
        out = torch.zeros(((R + T - 1) // T) * T * K, dtype=torch.float64, device="cuda")
        skgemm.pack_dev(R, K, dev(X), K, 1, T, out)   # row-major source
        assert np.array_equal(host(out), oracle.pack(X, T).ravel())
        out2 = torch.zeros_like(out)
        skgemm.pack_dev(R, K, dev(np.ascontiguousarray(X.T)), 1, R, T, out2)  # column-major
        assert np.array_equal(host(out2), oracle.pack(X, T).ravel())


def test_unpack_device_inverts_pack(cuda):
    R, K = 45, 70
    X = uniform((R, K), 9)
    for T in (16, 32):
        P = dev(oracle.pack(X, T))
        out = torch.full((R * K,), np.nan, dtype=torch.float64, device="cuda")
        skgemm.unpack_dev(R, K, P, T, out, K, 1)   # row-major destination
        assert np.array_equal(host(out).reshape(R, K), oracle.unpack(oracle.pack(X, T), R))
        out2 = torch.full((R * K,), np.nan, dtype=torch.float64, device="cuda")
        skgemm.unpack_dev(R, K, P, T, out2, 1, R)  # column-major destination
        assert np.array_equal(host(out2).reshape(K, R).T, X)


def test_linalg_c16_r16_converters(cuda):
    """linalg_pack_c16/r16 and unpack_c16/r16 (sme_pack.hpp:319-329): column-major
    [Nd, nb] = row-major [nb, Nd] bytes <-> grid-packed [Nd/16][nb][16]."""
    Nd, nb = 96, 40
    Psi = uniform((Nd, nb), 10)
    colmajor = dev(np.ascontiguousarray(Psi.T))  # src[g + b*Nd]
    for pack, unpack in ((skgemm.pack_c16_dev, skgemm.unpack_c16_dev),
                         (skgemm.pack_r16_dev, skgemm.unpack_r16_dev)):
        grid = torch.full((Nd * nb,), np.nan, dtype=torch.float64, device="cuda")
        pack(Nd, nb, colmajor, grid)
        assert np.array_equal(host(grid), oracle.grid_pack(Psi).ravel())
        back = torch.full((Nd * nb,), np.nan, dtype=torch.float64, device="cuda")
        unpack(Nd, nb, grid, back)
        assert np.array_equal(host(back), host(colmajor).ravel())
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.pack_c16_dev(Nd + 8, nb, colmajor, grid)
    assert e.value.code == skgemm.ERR_INVALID_ARG


# ------------------------------------------------- full-size configuration
def _config2_inputs(Nd=110592, nb=512, seed=77):
    rng = np.random.default_rng(seed)
    Psi = rng.standard_normal((Nd, nb)) / np.sqrt(Nd)
    HPsi = rng.standard_normal((Nd, nb)) / np.sqrt(Nd)
    Q = rng.uniform(-1.0, 1.0, (nb, nb))
    return Psi, HPsi, Q


def test_config2_subspace_ops_full_size(cuda):
    """Psi 110592 x 512 (48^3 grid x 512 states): S = Psi^T Psi, Hs = Psi^T HPsi,
    Psi' = Psi Q, checked on sampled entries against Dot2 and by properties."""
    Nd, nb = 110592, 512
    Psi, HPsi, Q = _config2_inputs(Nd, nb)
    dPsi, dH, dQ = dev(Psi), dev(HPsi), dev(Q)
    band = torch.empty(Nd * nb, dtype=torch.float64, device="cuda")
    h32 = torch.empty(Nd * nb, dtype=torch.float64, device="cuda")
    grid = torch.empty(Nd * nb, dtype=torch.float64, device="cuda")
    skgemm.pack_dev(nb, Nd, dPsi, 1, nb, 16, band)   # band-packed Psi
    skgemm.pack_dev(nb, Nd, dH, 1, nb, 32, h32)      # 32-band-packed HPsi
    skgemm.pack_dev(Nd, nb, dPsi, nb, 1, 16, grid)   # grid-packed Psi
    S = torch.zeros((nb, nb), dtype=torch.float64, device="cuda")
    Hs = torch.zeros((nb, nb), dtype=torch.float64, device="cuda")
    Pn = torch.empty(Nd * nb, dtype=torch.float64, device="cuda")
    skgemm.dsyrk_packed_dev(Nd, nb, band, S, nb, 1.0, 0.0)
    skgemm.dgemm_packed_dev(nb, nb, Nd, band, h32, Hs)
    skgemm.drot_dev(Nd, nb, grid, dQ, Pn)
    skgemm.stream_status()
    S_h = host(S).T  # column-major buffer: S_h[m1, m2]
    Hs_h = host(Hs)
    rng = np.random.default_rng(3)
    n = 512
    ii = rng.integers(0, nb, n)
    jj = rng.integers(0, nb, n)
    lo, hi = np.minimum(ii, jj), np.maximum(ii, jj)
    refS = oracle.dot2_sampled(Psi, Psi, lo, hi, x_strides=(1, nb), y_strides=(nb, 1), K=Nd)
    assert oracle.rel_frobenius(S_h[lo, hi], refS) <= TOL
    refH = oracle.dot2_sampled(Psi, HPsi, ii, jj, x_strides=(1, nb), y_strides=(nb, 1), K=Nd)
    assert oracle.rel_frobenius(Hs_h[ii, jj], refH) <= TOL
    gg = rng.integers(0, Nd, n)
    bb = rng.integers(0, nb, n)
    refP = oracle.dot2_sampled(Psi, Q, gg, bb)
    P_h = host(Pn)
    got = P_h[(bb // 16) * Nd * 16 + gg * 16 + bb % 16]
    assert oracle.rel_frobenius(got, refP) <= TOL
    # Properties: S is the GEMM of Psi with itself on the upper triangle;
    # the rotation is linear in Q.
    S2 = torch.zeros((nb, nb), dtype=torch.float64, device="cuda")
    b32 = torch.empty(Nd * nb, dtype=torch.float64, device="cuda")
    skgemm.pack_dev(nb, Nd, dPsi, 1, nb, 32, b32)
    skgemm.dgemm_packed_dev(nb, nb, Nd, band, b32, S2)
    iu = np.triu_indices(nb)
    assert oracle.rel_frobenius(S_h[iu], host(S2)[iu]) <= 1e-14
    P2 = torch.empty_like(Pn)
    skgemm.drot_dev(Nd, nb, grid, dQ * 2.0, P2)
    skgemm.stream_status()
    assert np.array_equal(host(P2), 2.0 * P_h)


@pytest.mark.parametrize("K", [40000, 16384])
def test_host_calls_with_chunked_upload(cuda, K):
    """Host-pointer GEMM and SYRK with long reductions upload their operands
    in k-chunks and multiply chunk c while chunk c + 1 is copied (GEMM:
    partial outputs summed at the end; SYRK: beta on the first chunk, 1 after).
    Results within 1e-13 of Dot2; SYRK's strict lower triangle comes back as
    passed."""
    M, N = 200, 136
    A, B = uniform((M, K), 5), uniform((K, N), 6)
    D = np.zeros(M * N)
    skgemm.gemm.compute_packed(M, N, K, oracle.pack(A, 16).ravel(),
                               oracle.pack(np.ascontiguousarray(B.T), 32).ravel(), D, 1.5, -0.25)
    ref = oracle.dot2_matmul(A, B, 1.5, -0.25)
    assert oracle.rel_frobenius(D.reshape(M, N), ref) <= TOL
    X = gaussian((K, M), 7, 1.0 / np.sqrt(K))
    C0 = uniform((M, M), 8)                     # column-major C: C0[j, i] = C(i, j)
    C = C0.ravel().copy()
    skgemm.sme_syrk.compute(K, M, oracle.pack(X.T, 16).ravel(), C, 2.0, 0.5)
    Cm = C.reshape(M, M)
    S = oracle.dot2_matmul(X.T, X)
    iu = np.triu_indices(M)
    want = 2.0 * S[iu] + 0.5 * C0[iu[1], iu[0]]
    assert oracle.rel_frobenius(Cm[iu[1], iu[0]], want) <= TOL
    il = np.tril_indices(M, -1)
    assert np.array_equal(Cm[il[1], il[0]], C0[il[1], il[0]])
