"""The device H Psi producers (skgemm_stencil_ext_dev, skgemm_nloc_apply_dev)
against golden outputs of the reference's own kernels
(tests/golden/reference_hpsi.npz), bit for bit."""
import numpy as np
import pytest
import torch

import skgemm
from tests.golden import make_golden_hpsi as G
from tests.test_golden_hpsi_cpu import check

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("c", range(len(G.STENCIL_CASES)))
@pytest.mark.parametrize("T", [32, 16])
def test_stencil_device_equals_golden(cuda, c, T):
    ni, nj, nk, nb = G.STENCIL_CASES[c]
    ext, A = G.stencil_inputs(ni, nj, nk, nb)
    out = torch.zeros((nb + T - 1) // T * ni * nj * nk * T, dtype=torch.float64, device="cuda")
    skgemm.stencil_ext_dev(ni, nj, nk, nb, torch.from_numpy(ext).cuda(),
                           torch.from_numpy(A).cuda(), G.CX, G.CY, G.CZ, G.C0, out, T)
    skgemm.stream_status()
    check(f"stencil{c}_t{T}", out.cpu().numpy())


@pytest.mark.parametrize("c", range(len(G.NLOC_CASES)))
@pytest.mark.parametrize("T", [32, 16])
def test_nloc_device_equals_golden(cuda, c, T):
    K, nb, nrow, ncol, atoms, images, dv = G.NLOC_CASES[c]
    pj, psi16, base = G.nloc_inputs(K, nb, nrow, ncol, atoms, images, T)
    h = skgemm.NlocProjector(pj.nrow, pj.ncol, pj.atom, pj.offsets, pj.index, pj.chi, pj.gamma, K)
    out = torch.from_numpy(base.copy()).cuda()
    h.apply(nb, dv, torch.from_numpy(psi16).cuda(), out, T)
    skgemm.stream_status()
    h.close()
    check(f"nloc{c}_t{T}", out.cpu().numpy())
