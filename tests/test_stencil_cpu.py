"""The H Psi stencil's oracle (oracle.c, oracle_stencil_ext / oracle_halo_periodic)
pinned to the reference: its own kernels from include/stencil_extended_packed.hpp,
compiled in place with the SVE emulation (oracle/_ref/libref_stencil.so), and
the naive loop of stencil_extended_test.cpp restated with numpy. CPU only."""
import ctypes

import numpy as np
import pytest

import oracle

# 6th-order coefficients and shape of stencil_extended_test.cpp:129-146.
CX = [0.0, -1.0 / 12, 2.0 / 3, -2.5, 8.0 / 3, -1.0 / 4, 1.0 / 30]
C0 = -0.5
F = 6


def extended_case(ni, nj, nk, nb, seed):
    rng = np.random.default_rng(seed)
    nix, njx, nkx = ni + 2 * F, nj + 2 * F, nk + 2 * F
    S_full = rng.uniform(-1, 1, (nb, nkx, njx, nix))
    A = rng.uniform(-1, 1, ni * nj * nk) * 10
    tiles = (nb + 15) // 16
    ext = np.zeros((tiles * 16, nkx * njx * nix))
    ext[:nb] = S_full.reshape(nb, -1)
    ext = np.ascontiguousarray(ext.reshape(tiles, 16, -1).transpose(0, 2, 1)).ravel()
    return S_full, A, ext


def ref_call(name, ext, A, ni, nj, nk, nb, T, cx=CX, c0=C0):
    K = ni * nj * nk
    out = np.zeros((nb + T - 1) // T * K * T)
    c = np.array(cx, dtype=np.float64)
    getattr(oracle.ref("stencil"), name)(oracle.ptr(ext), oracle.ptr(out), oracle.ptr(A), ni,
                                          nj, nk, nb, F, oracle.ptr(c), oracle.ptr(c),
                                          oracle.ptr(c), ctypes.c_double(c0))
    return out


@pytest.mark.parametrize("ni,nj,nk,nb", [(12, 10, 8, 48), (7, 9, 6, 40), (16, 16, 16, 32)])
def test_oracle_equals_reference_sve_kernels(ni, nj, nk, nb):
    _, A, ext = extended_case(ni, nj, nk, nb, ni * nj + nb)
    assert np.array_equal(oracle.stencil_ext(ext, A, ni, nj, nk, nb, CX, CX, CX, C0, 32),
                          ref_call("ref_stencil_16to32", ext, A, ni, nj, nk, nb, 32))
    assert np.array_equal(oracle.stencil_ext(ext, A, ni, nj, nk, nb, CX, CX, CX, C0, 16),
                          ref_call("ref_stencil_16to16", ext, A, ni, nj, nk, nb, 16))


def test_oracle_close_to_naive_and_scalar():
    ni, nj, nk, nb = 12, 10, 8, 48
    S_full, A, ext = extended_case(ni, nj, nk, nb, 12345)
    mine = oracle.stencil_ext(ext, A, ni, nj, nk, nb, CX, CX, CX, C0, 32)
    K = ni * nj * nk
    got = oracle.unpack(mine.reshape(-1, K, 32), nb)
    naive = oracle.stencil_naive(S_full, A, ni, nj, nk, nb, CX, CX, CX, C0).reshape(nb, K)
    assert np.max(np.abs(got - naive)) < 1e-12  # the reference test's bar is 1e-10
    scalar = ref_call("ref_stencil_16to32_scalar", ext, A, ni, nj, nk, nb, 32)
    assert np.max(np.abs(mine - scalar)) < 1e-12


def test_halo_periodic_oracle_is_a_wrap():
    ni, nj, nk, nb = 9, 7, 8, 20
    rng = np.random.default_rng(3)
    X = rng.standard_normal((nb, nk, nj, ni))
    K = ni * nj * nk
    local = oracle.pack(np.ascontiguousarray(X.reshape(nb, K)), 16).ravel()
    ext = oracle.halo_periodic(local, ni, nj, nk, nb)
    want = np.pad(X, ((0, 0), (F, F), (F, F), (F, F)), mode="wrap").reshape(nb, -1)
    assert np.array_equal(oracle.unpack(ext.reshape(-1, want.shape[1], 16), nb), want)


def test_binding_rejects_short_coefficient_lists():
    """The binding checks that each axis has FDn + 1 coefficients before the
    library reads them (raised before any device work; null pointers)."""
    import skgemm

    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.stencil_ext_dev(8, 8, 8, 16, 0, 0, CX, CX[:6], CX, C0, 0)
    assert e.value.code == skgemm.ERR_INVALID_ARG
