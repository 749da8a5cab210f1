"""Exactness of the residue conversion's FP32 arithmetic, restated on the CPU
with exact integers (host logic; no GPU).

The conversion kernels (convert_tma_kernel / convert_local_kernel) split the
scaled integer X = rint(v 2^mu), |X| <= 2^gamma(L), into digits and compute
its symmetric residue modulo each odd modulus m <= 255 in FP32:
    S = d0 + sum_j d_j c_j          (FMA chain; every partial sum an integer)
    q = rint(S * fl(1/m))           (fmaf(S, inv, 1.5*2^23) - 1.5*2^23)
    r = S - q m                     (one FMA)
which is exact when every partial sum stays below 2^24 and |S| < 2^23
(|S| |fl(1/m) - 1/m| < 1/(2m)). Two digit sets are used: for L <= 15
moduli, three unsigned 14-bit digits and a signed top digit X >> 42 with
symmetric constants c_j = 2^(14 j) mod m in (-m/2, m/2); for L = 16, four
unsigned 12-bit digits and a signed X >> 48 with c_j in [0, m). This file
checks the bounds for every L and replays the arithmetic exactly on random
and extreme X."""
import math

import numpy as np
import pytest

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193]
MAGIC = 3 << 22  # 1.5 * 2^23


def gamma_for(L):
    lg = sum(math.log2(m) for m in MODULI[:L])
    return math.floor((lg - 2.1) / 2)


def digit_plan(L):
    """(widths of the unsigned digits, symmetric constants?)"""
    return ([14, 14, 14], True) if L <= 15 else ([12, 12, 12, 12], False)


def consts(m, widths, symmetric):
    out, shift = [], 0
    for w in widths:
        shift += w
        c = pow(2, shift, m)
        if symmetric and c > m // 2:
            c -= m
        out.append(c)
    return out


def f32_inv(m):
    """fl(1/m) as (integer mantissa I, exponent e): value I * 2^e exactly."""
    f = np.float32(1.0) / np.float32(m)
    mant, ex = math.frexp(float(f))
    I = int(mant * (1 << 24))
    return I, ex - 24


def digits(X, widths):
    ds, rest = [], X.copy()
    for w in widths:
        ds.append(rest & ((1 << w) - 1))
        rest = rest >> w  # arithmetic shift: the top digit keeps the sign
    ds.append(rest)
    return ds


@pytest.mark.parametrize("L", range(6, 17))
def test_bounds_hold(L):
    g = gamma_for(L)
    widths, sym = digit_plan(L)
    top = 1 << max(g - sum(widths), 0)  # |X| <= 2^g => |X >> B| <= max(2^(g - B), 1)
    for m in MODULI[1:L]:
        c = consts(m, widths, sym)
        S_max = ((1 << widths[0]) - 1) + sum(abs(cj) * ((1 << w) - 1)
                                             for cj, w in zip(c[:-1], widths[1:])) \
            + abs(c[-1]) * top
        assert S_max < (1 << 23), (L, m, S_max)


@pytest.mark.parametrize("L", [6, 13, 14, 15, 16])
def test_replay_is_exact(L):
    g = gamma_for(L)
    widths, sym = digit_plan(L)
    rng = np.random.default_rng(L)
    lim = 1 << g
    X = np.concatenate([
        rng.integers(-lim, lim, 200000, dtype=np.int64, endpoint=True),
        np.array([lim, -lim, lim - 1, -lim + 1, 0, 1, -1], dtype=np.int64),
        rng.integers(-(1 << 20), 1 << 20, 20000, dtype=np.int64),
    ])
    ds = digits(X, widths)
    for m in MODULI[1:L]:
        c = consts(m, widths, sym)
        S = ds[0].copy()
        for cj, dj in zip(c, ds[1:]):
            S = S + cj * dj
            assert np.abs(S).max() < (1 << 24)  # every FMA partial sum exact in FP32
        I, e = f32_inv(m)
        prod = S * I  # S * fl(1/m) = prod * 2^e exactly (|prod| < 2^48)
        sh = -e
        # round-half-even of prod / 2^sh
        q = np.floor_divide(prod, 1 << sh)
        rem = prod - q * (1 << sh)
        half = 1 << (sh - 1)
        q = q + ((rem > half) | ((rem == half) & (q % 2 == 1))).astype(np.int64)
        r = S - q * m
        assert np.all(np.abs(r) <= (m - 1) // 2)
        assert np.array_equal(np.mod(r, m), np.mod(X, m)), (L, m)
