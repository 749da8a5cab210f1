"""The nonlocal projector on device (skgemm_nloc_create / _apply_dev) against
the oracle (itself equal to the reference's nloc_packed_opt2.hpp bit for bit,
tests/test_nloc_cpu.py), bit for bit."""
import numpy as np
import pytest
import torch

import oracle
import skgemm
from tests.test_nloc_cpu import CASES

pytestmark = pytest.mark.gpu


def handle(pj, K):
    return skgemm.NlocProjector(pj.nrow, pj.ncol, pj.atom, pj.offsets, pj.index, pj.chi,
                                pj.gamma, K)


@pytest.mark.parametrize("K,nb,nrow,ncol,P,images", CASES + [(20000, 100, 700, 16, 12, 4)])
@pytest.mark.parametrize("T", [32, 16])
def test_nloc_equals_oracle(cuda, K, nb, nrow, ncol, P, images, T):
    pj = oracle.nloc_random(K, nrow, ncol, P, seed=K + nb + images, images=images)
    rng = np.random.default_rng(K + 1)
    psi16 = rng.uniform(-1, 1, (nb + 15) // 16 * K * 16)
    base = rng.uniform(-1, 1, (nb + T - 1) // T * K * T)
    want = oracle.nloc_project(pj, psi16, nb, K, 0.01, base.copy(), T)
    h = handle(pj, K)
    out = torch.from_numpy(base.copy()).cuda()
    h.apply(nb, 0.01, torch.from_numpy(psi16).cuda(), out, T)
    skgemm.stream_status()
    assert np.array_equal(out.cpu().numpy(), want)
    h.close()


def test_nloc_handle_reused_across_band_counts(cuda):
    """One handle applied at growing band counts (its scratch regrows) and
    twice at the same count (out accumulates): each call equals the oracle."""
    K = 5000
    pj = oracle.nloc_random(K, 300, 9, 6, seed=77, images=2)
    h = handle(pj, K)
    rng = np.random.default_rng(5)
    for nb in (16, 200, 40, 200):
        psi16 = rng.uniform(-1, 1, (nb + 15) // 16 * K * 16)
        base = rng.uniform(-1, 1, (nb + 31) // 32 * K * 32)
        want = oracle.nloc_project(pj, psi16, nb, K, 0.03, base.copy(), 32)
        want = oracle.nloc_project(pj, psi16, nb, K, 0.03, want, 32)
        out = torch.from_numpy(base.copy()).cuda()
        p = torch.from_numpy(psi16).cuda()
        h.apply(nb, 0.03, p, out, 32)
        h.apply(nb, 0.03, p, out, 32)
        skgemm.stream_status()
        assert np.array_equal(out.cpu().numpy(), want), nb
    h.close()


def test_nloc_repeated_atoms_and_empty_projectors(cuda):
    """Atoms that come back after another atom (scaled again, as the
    reference's change-of-atom rule does) and projectors without rows."""
    K, nb = 3000, 48
    pj = oracle.nloc_random(K, 90, 7, 3, seed=9, images=2)
    atom = pj.atom.copy()
    atom[[1, 3, 5]] = atom[[0, 2, 4]] + 1  # images interleaved with the next atom
    nrow = pj.nrow.copy()
    nrow[2] = 0  # a projector without rows (its rows dropped from index / chi)
    keep_rows = np.concatenate([np.arange(pj.row_off[p], pj.row_off[p] + pj.nrow[p])
                                for p in range(len(nrow)) if nrow[p]])
    keep_chi = np.concatenate([np.arange(pj.chi_off[p], pj.chi_off[p] + pj.nrow[p] * pj.ncol[p])
                               for p in range(len(nrow)) if nrow[p]])
    pj2 = oracle.NlocProjectors(nrow, pj.ncol, atom, pj.offsets, pj.index[keep_rows],
                                pj.chi[keep_chi], pj.gamma)
    rng = np.random.default_rng(2)
    psi16 = rng.uniform(-1, 1, (nb + 15) // 16 * K * 16)
    want = oracle.nloc_project(pj2, psi16, nb, K, 0.02, np.zeros((nb + 31) // 32 * K * 32), 32)
    out = torch.zeros((nb + 31) // 32 * K * 32, dtype=torch.float64, device="cuda")
    h = handle(pj2, K)
    h.apply(nb, 0.02, torch.from_numpy(psi16).cuda(), out, 32)
    skgemm.stream_status()
    assert np.array_equal(out.cpu().numpy(), want)


def test_nloc_rejects_bad_sets(cuda):
    pj = oracle.nloc_random(100, 10, 4, 2, seed=1)
    with pytest.raises(skgemm.SkgemmError):  # index past K
        skgemm.NlocProjector(pj.nrow, pj.ncol, pj.atom, pj.offsets, pj.index + 100, pj.chi,
                             pj.gamma, 100)
    off = pj.offsets.copy()
    off[1] = 2  # overlapping blocks
    with pytest.raises(skgemm.SkgemmError):
        skgemm.NlocProjector(pj.nrow, pj.ncol, pj.atom, off, pj.index, pj.chi, pj.gamma, 100)
