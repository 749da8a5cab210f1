"""The nonlocal projector's oracle (oracle_nloc_project) pinned to the
reference's own include/nloc_packed_opt2.hpp, compiled in place through its
test file (oracle/_ref/libref_nloc.so). CPU only."""
import ctypes

import numpy as np
import pytest

import oracle

# (K, nb, nrow, ncol, projectors) of nloc_packed_opt2_test.cpp:292-296, plus
# shared-atom (periodic image) and ragged-band cases.
CASES = [(100, 16, 20, 5, 1, 1), (200, 32, 50, 8, 2, 1), (500, 48, 100, 12, 3, 1),
         (1000, 64, 200, 16, 2, 1), (2000, 128, 300, 20, 4, 1), (1500, 40, 120, 9, 3, 3)]


def ref_project(pj, psi16, nb, K, dv, out, T):
    c = ctypes
    a = pj.args()
    oracle.ref("nloc").ref_nloc_project(
        c.c_int(a[0]), *a[1:6], pj.row_off.ctypes.data_as(c.POINTER(c.c_longlong)), a[7],
        pj.chi_off.ctypes.data_as(c.POINTER(c.c_longlong)), a[9],
        pj.gam_off.ctypes.data_as(c.POINTER(c.c_longlong)), c.c_int(nb), c.c_int(K),
        c.c_double(dv), oracle.ptr(psi16), oracle.ptr(out), c.c_int(T))
    return out


@pytest.mark.parametrize("K,nb,nrow,ncol,P,images", CASES)
@pytest.mark.parametrize("T", [32, 16])
def test_oracle_equals_reference(K, nb, nrow, ncol, P, images, T):
    pj = oracle.nloc_random(K, nrow, ncol, P, seed=K + nb + images, images=images)
    rng = np.random.default_rng(K)
    psi16 = rng.uniform(-1, 1, (nb + 15) // 16 * K * 16)
    base = rng.uniform(-1, 1, (nb + T - 1) // T * K * T)
    mine = oracle.nloc_project(pj, psi16, nb, K, 0.01, base.copy(), T)
    ref = ref_project(pj, psi16, nb, K, 0.01, base.copy(), T)
    assert np.array_equal(mine, ref)


def test_projector_host_arrays_checked():
    """The binding rejects host arrays shorter than the set they describe
    before the library reads them (no device needed)."""
    import skgemm

    pj = oracle.nloc_random(100, 10, 4, 2, seed=3)
    args = [pj.nrow, pj.ncol, pj.atom, pj.offsets, pj.index, pj.chi, pj.gamma]
    bad = [(3, pj.offsets[:-1]), (4, pj.index[:-1]), (5, pj.chi[:-1]), (6, pj.gamma[:-1]),
           (1, pj.ncol[:-1]), (2, pj.atom[:-1])]
    for pos, arr in bad:
        a = list(args)
        a[pos] = arr
        with pytest.raises(skgemm.SkgemmError) as e:
            skgemm.NlocProjector(*a, 100)
        assert e.value.code == skgemm.ERR_INVALID_ARG
