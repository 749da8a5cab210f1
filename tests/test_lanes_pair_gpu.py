"""The CTA-pair (tcgen05 .cta_group::2) lanes kernel against the one-CTA
kernel: both write the same int32 partial slabs, so every Ozaki GEMM, SYRK,
subspace pair and the exact int8 GEMM must agree bit for bit (the rotations,
whose products run on the one-CTA B-resident kernel either way, are checked
alongside). The one-CTA
results come from a child process with SKGEMM_LANES_PAIR=0 (the switch is
read once per process); this process runs the default (pair) kernel."""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import oracle
import skgemm

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [(512, 512, 110592), (300, 200, 4099), (1, 513, 77), (640, 384, 20000),
         (257, 33, 140000)]


def compute(prec):
    """Results of the lanes products for CASES, as numpy arrays."""
    out = []
    for i, (M, N, K) in enumerate(CASES):
        g = torch.Generator(device="cuda").manual_seed(100 + i)
        X = torch.randn(K, M, generator=g, dtype=torch.float64, device="cuda") / K ** 0.5
        Y = torch.randn(K, N, generator=g, dtype=torch.float64, device="cuda") / K ** 0.5
        P16 = torch.empty(((M + 15) // 16) * 16 * K, dtype=torch.float64, device="cuda")
        P32 = torch.empty(((N + 31) // 32) * 32 * K, dtype=torch.float64, device="cuda")
        skgemm.pack_dev(M, K, X, 1, M, 16, P16)
        skgemm.pack_dev(N, K, Y, 1, N, 32, P32)
        D = torch.zeros(M * N, dtype=torch.float64, device="cuda")
        C = torch.zeros(M * M, dtype=torch.float64, device="cuda")
        skgemm.dgemm_packed_dev(M, N, K, P16, P32, D, N, 1.25, -0.5, precision=prec)
        skgemm.dsyrk_packed_dev(K, M, P16, C, M, precision=prec)
        res = [D.cpu().numpy(), C.cpu().numpy()]
        if M == N:
            P32b = torch.empty(((M + 31) // 32) * 32 * K, dtype=torch.float64, device="cuda")
            skgemm.pack_dev(M, K, Y, 1, M, 32, P32b)
            S = torch.zeros(M * M, dtype=torch.float64, device="cuda")
            Hs = torch.zeros(M * M, dtype=torch.float64, device="cuda")
            skgemm.dsubspace_packed_dev(K, M, P16, P32b, S, Hs, precision=prec)
            res += [S.cpu().numpy(), Hs.cpu().numpy()]
        skgemm.stream_status()
        out.append(res)
    # Rotations, one of them with an odd number of 128-row tiles.
    for j, (Nd, nb) in enumerate([(4096, 512), (12288, 256), (1040, 208), (110592, 512)]):
        g = torch.Generator(device="cuda").manual_seed(200 + j)
        Psi = torch.randn(Nd, nb, generator=g, dtype=torch.float64, device="cuda") / Nd ** 0.5
        Q = torch.rand(nb, nb, generator=g, dtype=torch.float64, device="cuda") * 2 - 1
        G = torch.empty(Nd * nb, dtype=torch.float64, device="cuda")
        skgemm.pack_dev(Nd, nb, Psi, nb, 1, 16, G)
        R = torch.full((Nd * nb,), float("nan"), dtype=torch.float64, device="cuda")
        if prec == skgemm.PREC_OZAKI_BF16 and nb > 1024:
            continue
        skgemm.drot_dev(Nd, nb, G, Q, R, precision=prec)
        skgemm.stream_status()
        out.append([R.cpu().numpy()])
    ai = torch.randint(-128, 128, (700, 3000), dtype=torch.int8, device="cuda",
                       generator=torch.Generator(device="cuda").manual_seed(7))
    bi = torch.randint(-128, 128, (333, 3000), dtype=torch.int8, device="cuda",
                       generator=torch.Generator(device="cuda").manual_seed(8))
    ci = torch.zeros(700, 333, dtype=torch.int32, device="cuda")
    skgemm.igemm_s8_dev(700, 333, 3000, ai, 3000, bi, 3000, ci, 333)
    skgemm.stream_status()
    out.append([ci.cpu().numpy()])
    return out


def _flat(out):
    return [a for res in out for a in res]


@pytest.mark.parametrize("prec", [skgemm.PREC_OZAKI_I8, skgemm.PREC_OZAKI_BF16])
def test_pair_kernel_equals_one_cta_kernel(cuda, tmp_path, prec):
    path = str(tmp_path / "one_cta.npz")
    code = (f"import sys; sys.path[:0] = [{REPO!r}, {os.path.join(REPO, 'stream-k-gemm_b200')!r}]\n"
            "import numpy as np\n"
            "from tests.test_lanes_pair_gpu import compute, _flat\n"
            f"np.savez({path!r}, *_flat(compute({prec})))\n")
    env = dict(os.environ, SKGEMM_LANES_PAIR="0")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = np.load(path)
    got = _flat(compute(prec))
    assert len(got) == len(ref.files)
    for k, a in enumerate(got):
        assert np.array_equal(a, ref[f"arr_{k}"]), k


def test_pair_kernel_ozaki_gemm_accuracy(cuda):
    """The pair kernel's GEMM at the subspace size against sampled Dot2."""
    M = N = 512
    K = 110592
    rng = np.random.default_rng(3)
    A = rng.standard_normal((M, K)) / np.sqrt(K)
    B = rng.standard_normal((K, N)) / np.sqrt(K)
    D = torch.zeros(M * N, dtype=torch.float64, device="cuda")
    skgemm.dgemm_packed_dev(M, N, K, torch.from_numpy(oracle.pack(A, 16)).cuda(),
                            torch.from_numpy(oracle.pack(np.ascontiguousarray(B.T), 32)).cuda(),
                            D, N, precision=skgemm.PREC_OZAKI_I8)
    skgemm.stream_status()
    ii, jj = rng.integers(0, M, 2048), rng.integers(0, N, 2048)
    ref = oracle.dot2_sampled(A, B, ii, jj)
    assert oracle.rel_frobenius(D.cpu().numpy().reshape(M, N)[ii, jj], ref) <= 1e-13
