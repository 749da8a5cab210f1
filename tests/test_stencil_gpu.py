"""The H Psi producer on device (skgemm_stencil_ext_dev, skgemm_halo_periodic_dev):
bit for bit against the oracle (itself equal to the reference's SVE kernels,
tests/test_stencil_cpu.py), and feeding Hs = Psi^T (H Psi) through the GEMM."""
import numpy as np
import pytest
import torch

import oracle
import skgemm
from tests.test_stencil_cpu import C0, CX, F, extended_case

pytestmark = pytest.mark.gpu


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).to("cuda")


@pytest.mark.parametrize("ni,nj,nk,nb", [(12, 10, 8, 48), (13, 7, 9, 40), (16, 16, 16, 32),
                                         (33, 5, 20, 17), (48, 48, 48, 64)])
@pytest.mark.parametrize("T", [32, 16])
def test_stencil_equals_oracle(cuda, ni, nj, nk, nb, T):
    _, A, ext = extended_case(ni, nj, nk, nb, 7 * ni + nb)
    K = ni * nj * nk
    CY = [0.0] + [c * 0.75 for c in CX[1:]]
    CZ = [0.0] + [c * 1.25 for c in CX[1:]]
    out = torch.full(((nb + T - 1) // T * K * T,), np.nan, dtype=torch.float64, device="cuda")
    skgemm.stencil_ext_dev(ni, nj, nk, nb, dev(ext), dev(A), CX, CY, CZ, C0, out, T)
    skgemm.stream_status()
    want = oracle.stencil_ext(ext, A, ni, nj, nk, nb, CX, CY, CZ, C0, T, threads=oracle.nthreads())
    got = out.cpu().numpy()
    lanes = np.arange(got.size) % T + (np.arange(got.size) // (K * T)) * T
    assert np.array_equal(got[lanes < nb], want[lanes < nb])
    assert np.isnan(got[lanes >= nb]).all()  # padding lanes untouched


def test_halo_periodic_equals_oracle(cuda):
    ni, nj, nk, nb = 24, 20, 16, 40
    rng = np.random.default_rng(11)
    local = rng.standard_normal((nb + 15) // 16 * ni * nj * nk * 16)
    ext = torch.full((oracle.ext_size(ni, nj, nk, nb),), np.nan, dtype=torch.float64, device="cuda")
    skgemm.halo_periodic_dev(ni, nj, nk, nb, dev(local), ext)
    skgemm.stream_status()
    assert np.array_equal(ext.cpu().numpy(), oracle.halo_periodic(local, ni, nj, nk, nb))


def test_stencil_feeds_hs(cuda):
    """Psi (band-packed) -> periodic halo -> H Psi (32-band-packed) -> Hs =
    Psi^T H Psi with the GEMM, all on the device; against Dot2 of the oracle's
    H Psi."""
    ni = nj = nk = 24
    nb = 96
    K = ni * nj * nk
    rng = np.random.default_rng(5)
    psi = rng.standard_normal((K, nb)) / np.sqrt(K)
    A = rng.uniform(-1, 1, K)
    band = oracle.band_pack(psi).ravel()
    ext = torch.empty(oracle.ext_size(ni, nj, nk, nb), dtype=torch.float64, device="cuda")
    skgemm.halo_periodic_dev(ni, nj, nk, nb, dev(band), ext)
    hpsi = torch.zeros(K * nb, dtype=torch.float64, device="cuda")
    skgemm.stencil_ext_dev(ni, nj, nk, nb, ext, dev(A), CX, CX, CX, C0, hpsi, 32)
    Hs = torch.zeros(nb * nb, dtype=torch.float64, device="cuda")
    skgemm.dgemm_packed_dev(nb, nb, K, dev(band), hpsi, Hs, nb)
    skgemm.stream_status()
    h32 = oracle.stencil_ext(oracle.halo_periodic(band, ni, nj, nk, nb), A, ni, nj, nk, nb,
                             CX, CX, CX, C0, 32)
    hdense = oracle.unpack(h32.reshape(-1, K, 32), nb).T  # (K, nb)
    assert np.array_equal(hpsi.cpu().numpy(), h32)
    ref = oracle.dot2_matmul(np.ascontiguousarray(psi.T), hdense)
    assert oracle.rel_frobenius(Hs.cpu().numpy().reshape(nb, nb), ref) <= 1e-13


def test_stencil_rejects_other_radius(cuda):
    x = torch.zeros(16 * 32 ** 3, dtype=torch.float64, device="cuda")
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.stencil_ext_dev(8, 8, 8, 16, x, x, CX[:5], CX[:5], CX[:5], C0, x, 32, FDn=4)
    assert e.value.code == skgemm.ERR_UNSUPPORTED
