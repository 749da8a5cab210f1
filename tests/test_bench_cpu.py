"""CPU checks of bench.py's in-run accuracy leg: the double-double products
(dd_products) that rate S, Hs and Psi' against an extended-precision
reference, and the index maps (column-major S, row-major Hs, band-packed
Psi') that subspace_errors reads. Checked against the oracle's Dot2 and on a
cancellation plain FP64 gets wrong; a planted error is seen."""
import numpy as np
import torch

import bench
import oracle


def test_dd_products_match_dot2_and_survive_cancellation():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((5000, 7))
    Y = rng.standard_normal((5000, 5))
    got = bench.dd_products(torch.from_numpy(X), torch.from_numpy(Y), chunk=1024).numpy()
    ref = oracle.dot2_matmul(X.T, Y)
    assert np.max(np.abs(got - ref) / np.abs(ref)) <= 4e-16
    x = torch.tensor([[1e16], [1.0], [-1e16], [3.0]], dtype=torch.float64)
    y = torch.ones(4, 1, dtype=torch.float64)
    assert (x.T @ y).item() != 4.0                 # plain FP64 loses the 1
    assert bench.dd_products(x, y).item() == 4.0


def test_subspace_errors_index_maps():
    nd, nb = 512, 64
    bench.set_shape(nd, nb)
    try:
        g = torch.Generator().manual_seed(1)
        psi = torch.randn(nd, nb, generator=g, dtype=torch.float64)
        hpsi = torch.randn(nd, nb, generator=g, dtype=torch.float64)
        q = torch.rand(nb, nb, generator=g, dtype=torch.float64)
        st = torch.tensor([0, 5, 17, 63])
        gs = torch.tensor([1, 100, 511])
        check = {"st": st, "gs": gs, "psi_cols": psi[:, st].contiguous(),
                 "hpsi_cols": hpsi[:, st].contiguous(), "psi_rows": psi[gs].contiguous(),
                 "q": q}
        S = (psi.T @ psi).T.contiguous()            # column-major: S[i + j nb] = S(i, j)
        Hs = (psi.T @ hpsi).contiguous()
        P = psi @ q
        Pn = torch.from_numpy(oracle.band_pack(P.numpy()).ravel().copy())
        e = bench.subspace_errors(S, Hs, Pn, check)
        assert max(e.values()) <= 1e-14, e
        S.view(-1)[5 + 17 * nb] += 1e-6            # S(5, 17): in the sampled upper triangle
        Pn.view(nb // 16, nd, 16)[17 // 16, 100, 17 % 16] += 1e-6
        e = bench.subspace_errors(S, Hs, Pn, check)
        assert e["S"] > 1e-10 and e["Psi_Q"] > 1e-10 and e["Hs"] <= 1e-14
    finally:
        bench.set_shape(bench.ND0, bench.NB0)


def test_profile_traffic_lines_parse():
    """The bench's `roofline.traffic` comes from the committed ncu summaries'
    `traffic_bytes_per_launch <kernel>:` lines: each kernel the headline
    roofline can name has one, and it parses to bytes per launch."""
    for kernel, lo, hi in [("convert_tma_kernel", 1e9, 2e9),
                           ("i8_gemm2_kernel", 5e8, 2e9),
                           ("i8_rot_kernel", 1e9, 2e9),
                           ("fp64_streamk_kernel", 1e9, 4e9),
                           ("fp64_streamk_kernel64", 1e9, 4e9),
                           ("stencil_staged_kernel", 1e9, 2e9),
                           ("nloc_backward_kernel", 5e8, 2e9)]:
        t = bench.read_profile_traffic(kernel)
        assert t is not None and lo <= t <= hi, (kernel, t)
    assert bench.read_profile_traffic("no_such_kernel") is None
