"""The allocation-free packed GEMM entry point, called through the C ABI.

skgemm_dgemm_packed_dev_noalloc serves callers that cannot allocate device
memory when they call the GEMM (their memory is reserved in their own pool,
or their device footprint must stay fixed after start-up): its Stream-K
scratch is a static device array instead of a workspace allocated on first
use. These tests check that it returns what the regular entry point
(skgemm_dgemm_packed_dev) returns, on two calls in a row with different
shapes (the second finds the first's leftovers in the shared scratch), and
that a call on a fresh stream leaves the device's free memory unchanged.

This file is collected last so that a run stopping at the first failure has
run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import skgemm

pytestmark = pytest.mark.gpu
TOL = 1e-13  # relative Frobenius tolerance used by the parity tests


def _noalloc(M, N, K, Ap, Bp, D, ldd, alpha, gamma, stream=0):
    f = skgemm.lib().skgemm_dgemm_packed_dev_noalloc
    rc = f(M, N, K, ctypes.c_void_p(Ap.data_ptr()), ctypes.c_void_p(Bp.data_ptr()),
           ctypes.c_void_p(D.data_ptr()), ldd, alpha, gamma, ctypes.c_void_p(stream))
    if rc != 0:
        raise skgemm.SkgemmError(rc, skgemm.lib().skgemm_last_error().decode())


def _operands(M, N, K, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    Ap = torch.from_numpy(oracle.pack(A, 16)).cuda()
    Bp = torch.from_numpy(oracle.pack(np.ascontiguousarray(B.T), 32)).cuda()
    return Ap, Bp


@pytest.mark.parametrize("M,N,K,alpha,gamma", [(512, 512, 65536, 1.0, 0.0),
                                               (333, 129, 4099, -1.5, 0.25)])
def test_noalloc_matches_regular_entry_two_calls(cuda, M, N, K, alpha, gamma):
    Ap, Bp = _operands(M, N, K, M + K)
    ref = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
    skgemm.dgemm_packed_dev(M, N, K, Ap, Bp, ref, N, alpha, gamma)
    skgemm.stream_status()
    for _ in range(2):
        out = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
        _noalloc(M, N, K, Ap, Bp, out, N, alpha, gamma)
        torch.cuda.synchronize()
        assert oracle.rel_frobenius(out.cpu().numpy(), ref.cpu().numpy()) <= TOL
        assert not torch.isnan(out).any()


def test_noalloc_new_stream_allocates_nothing(cuda):
    M, N, K = 256, 384, 20000
    Ap, Bp = _operands(M, N, K, 9)
    out = torch.zeros((M, N), dtype=torch.float64, device="cuda")
    ref = torch.zeros_like(out)
    _noalloc(M, N, K, Ap, Bp, out, N, 1.0, 0.0)  # first call on the device: set-up
    skgemm.dgemm_packed_dev(M, N, K, Ap, Bp, ref, N, 1.0, 0.0)
    skgemm.stream_status()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    _noalloc(M, N, K, Ap, Bp, out, N, 1.0, 0.0, stream=s.cuda_stream)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert oracle.rel_frobenius(out.cpu().numpy(), ref.cpu().numpy()) <= TOL


def test_noalloc_rejects_bad_arguments(cuda):
    d = torch.zeros(64, dtype=torch.float64, device="cuda")
    with pytest.raises(skgemm.SkgemmError) as e:
        _noalloc(4, 8, 16, d, d, d, 4, 1.0, 0.0)  # ldd < N
    assert e.value.code == skgemm.ERR_INVALID_ARG
