"""The failure path of the device-side waits, exercised without a fault: a
bounded wait on an mbarrier that nothing arrives on runs out after its
budget; the kernel records the timeout in the stream's device error word and
returns; skgemm_stream_status reports SKGEMM_ERR_DEVICE_TIMEOUT once and
clears the word; the GPU context keeps working (a GEMM on the same stream is
correct afterwards)."""
import time

import numpy as np
import pytest
import torch

import oracle
import skgemm
from tests._cases import uniform

pytestmark = pytest.mark.gpu


def test_expired_wait_is_reported_and_the_context_survives(cuda):
    s = torch.cuda.Stream()
    t0 = time.perf_counter()
    skgemm.diag_expire_wait(50.0, stream=s)
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.stream_status(s)
    assert e.value.code == skgemm.ERR_DEVICE_TIMEOUT
    assert time.perf_counter() - t0 >= 0.045      # the wait lasted its budget
    skgemm.stream_status(s)                       # reported once, then cleared
    M, N, K = 96, 80, 700
    A, B = uniform((M, K), 1), uniform((K, N), 2)
    dA = torch.from_numpy(oracle.pack(A, 16).ravel()).cuda()
    dB = torch.from_numpy(oracle.pack(np.ascontiguousarray(B.T), 32).ravel()).cuda()
    D = torch.zeros(M * N, dtype=torch.float64, device="cuda")
    with torch.cuda.stream(s):
        skgemm.dgemm_packed_dev(M, N, K, dA, dB, D, N, 1.0, 0.0, stream=s)
    skgemm.stream_status(s)
    err = oracle.rel_frobenius(D.cpu().numpy().reshape(M, N), oracle.dot2_matmul(A, B))
    assert err <= 1e-13


def test_expire_wait_rejects_bad_budgets(cuda):
    for b in (0.0, -1.0, 5000.0):
        with pytest.raises(skgemm.SkgemmError):
            skgemm.diag_expire_wait(b)


def test_expired_fixup_wait_is_reported_and_the_context_survives(cuda):
    """The Stream-K fixup's flag wait (the CTA finishing a tile waiting for a
    later CTA's partial) runs out on a flag nothing sets: the timeout is
    recorded as the fixup's code (error word 0x2), reported once, and a
    Stream-K GEMM whose tiles are split across CTAs is correct afterwards on
    the same stream."""
    s = torch.cuda.Stream()
    t0 = time.perf_counter()
    skgemm.diag_expire_fixup_wait(50.0, stream=s)
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.stream_status(s)
    assert e.value.code == skgemm.ERR_DEVICE_TIMEOUT
    assert "0x2)" in str(e.value)                 # kDevErrFixupTimeout
    assert time.perf_counter() - t0 >= 0.045
    skgemm.stream_status(s)
    M, N, K = 256, 256, 60000                     # 4 tiles over many CTAs: fixups
    A, B = uniform((M, K), 3), uniform((K, N), 4)
    dA = torch.from_numpy(oracle.pack(A, 16).ravel()).cuda()
    dB = torch.from_numpy(oracle.pack(np.ascontiguousarray(B.T), 32).ravel()).cuda()
    D = torch.zeros(M * N, dtype=torch.float64, device="cuda")
    with torch.cuda.stream(s):
        skgemm.dgemm_packed_dev(M, N, K, dA, dB, D, N, 1.0, 0.0, stream=s)
    skgemm.stream_status(s)
    err = oracle.rel_frobenius(D.cpu().numpy().reshape(M, N), oracle.dot2_matmul(A, B))
    assert err <= 1e-13


def test_expire_fixup_wait_rejects_bad_budgets(cuda):
    for b in (0.0, -1.0, 5000.0):
        with pytest.raises(skgemm.SkgemmError):
            skgemm.diag_expire_fixup_wait(b)
