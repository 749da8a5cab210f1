"""Shared input generators: the reference's known-answer inputs and the seeded
synthetic workloads (uniform / Gaussian / exponent-stress entries)."""
from __future__ import annotations

import numpy as np

import oracle
from tests.golden.make_golden import GEMM_CASES, ROT_CASES, SYRK_CASES, gemm_inputs, rot_inputs  # noqa: F401


def uniform(shape, seed, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, size=shape)


def gaussian(shape, seed, scale=1.0):
    return np.random.default_rng(seed).standard_normal(size=shape) * scale


def stress(shape, seed, emin=-20, emax=20):
    """sign * 2^e * m, e uniform integer in [emin, emax], m uniform in [1, 2)."""
    rng = np.random.default_rng(seed)
    sign = rng.choice([-1.0, 1.0], size=shape)
    e = rng.integers(emin, emax + 1, size=shape)
    m = rng.uniform(1.0, 2.0, size=shape)
    return sign * np.ldexp(m, e)


def golden_check(golden, key, values, rtol=1e-9):
    """Compare a full output (flattened like the golden's producer) against a
    golden entry: the sampled/whole entries and the global checksums."""
    v = np.ascontiguousarray(values, dtype=np.float64).ravel()
    assert v.size == int(golden[f"{key}_size"][0]), (v.size, golden[f"{key}_size"])
    idx = golden[f"{key}_idx"]
    ref = golden[f"{key}_val"]
    scale = np.maximum(1.0, np.abs(ref))
    err = np.max(np.abs(v[idx] - ref) / scale)
    assert err <= rtol, f"{key}: max scaled error {err:.3e} > {rtol}"
    s, ss = v.sum(), (v * v).sum()
    assert abs(s - golden[f"{key}_sum"][0]) <= rtol * max(1.0, abs(golden[f"{key}_sum"][0])) * 10
    assert abs(ss - golden[f"{key}_sumsq"][0]) <= rtol * max(1.0, golden[f"{key}_sumsq"][0]) * 10
    return err
