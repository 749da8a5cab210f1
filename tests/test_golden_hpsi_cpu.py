"""The H Psi oracles against golden outputs of the reference's own kernels
(tests/golden/reference_hpsi.npz, made by tests/golden/make_golden_hpsi.py from
the stencil and projector kernels compiled in place): bit for bit, without the
reference tree. CPU only."""
import os

import numpy as np
import pytest

import oracle
from tests.golden import make_golden_hpsi as G

GOLD = np.load(os.path.join(os.path.dirname(G.__file__), "reference_hpsi.npz"))


def check(key, got):
    got = np.ascontiguousarray(got).ravel()
    assert got.size == int(GOLD[f"{key}_size"][0])
    assert np.array_equal(got[GOLD[f"{key}_idx"]], GOLD[f"{key}_val"]), key
    assert got.sum() == pytest.approx(float(GOLD[f"{key}_sum"][0]), rel=1e-13, abs=1e-13)
    assert (got * got).sum() == pytest.approx(float(GOLD[f"{key}_sumsq"][0]), rel=1e-13)


@pytest.mark.parametrize("c", range(len(G.STENCIL_CASES)))
@pytest.mark.parametrize("T", [32, 16])
def test_stencil_oracle_equals_golden(c, T):
    ni, nj, nk, nb = G.STENCIL_CASES[c]
    ext, A = G.stencil_inputs(ni, nj, nk, nb)
    check(f"stencil{c}_t{T}", oracle.stencil_ext(ext, A, ni, nj, nk, nb, G.CX, G.CY, G.CZ,
                                                 G.C0, T))


@pytest.mark.parametrize("c", range(len(G.NLOC_CASES)))
@pytest.mark.parametrize("T", [32, 16])
def test_nloc_oracle_equals_golden(c, T):
    K, nb, nrow, ncol, atoms, images, dv = G.NLOC_CASES[c]
    pj, psi16, base = G.nloc_inputs(K, nb, nrow, ncol, atoms, images, T)
    check(f"nloc{c}_t{T}", oracle.nloc_project(pj, psi16, nb, K, dv, base, T))
