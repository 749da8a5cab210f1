"""GPU parity at the long reductions and large state counts of the batched
and serving configurations (grids up to 4e5 points, up to 2048 states).

The Ozaki path cuts K into segments of at most 1023 k-blocks per modulus
(INT32 exactness), so K > 130944 crosses segment boundaries; BF16 residues
add sub-segments of 16 k-blocks per FP32 accumulation. These tests pin the
segment-crossing and large-state code against the Dot2 (double-double)
oracle on sampled entries: relative Frobenius error <= 1e-13 over the
sample, for native FP64, Ozaki INT8 and Ozaki BF16, on Gaussian
N(0,1)/sqrt(K) and exponent-stress (sign * 2^e * m, e in [-20, 20]) inputs.

Inputs are drawn on the device from a seeded generator (dense, grid-major:
X[k][state]) and packed with skgemm_pack_dev (checked bit for bit against
the oracle's packing elsewhere); state-major copies go to the host for the
oracle. The reference handles any K (gemm_opt.cpp:255, syrk_crsp.cpp:355);
rotations follow sme_trp_3d.hpp:194 (nb a multiple of 32).
"""
import numpy as np
import pytest
import torch

import oracle
import skgemm

pytestmark = pytest.mark.gpu
TOL = 1e-13
NS = 2048  # sampled entries per result
I8, BF, NAT = skgemm.PREC_OZAKI_I8, skgemm.PREC_OZAKI_BF16, skgemm.PREC_NATIVE


@pytest.fixture(autouse=True)
def _release_device_memory():
    """These cases hold several GB each: return torch's cached blocks and the
    library's per-stream scratch after every case, so that later tests in the
    same process find the device's memory free."""
    yield
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    skgemm.stream_release(torch.cuda.current_stream())
    skgemm.stream_release(None)


def draw(kind, rows, cols, seed):
    """rows x cols float64 on the device: Gaussian N(0,1)/sqrt(rows) or the
    exponent stress sign * 2^e * m (e integer in [-20, 20], m in [1, 2))."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    if kind == "gauss":
        return torch.randn(rows, cols, generator=g, dtype=torch.float64, device="cuda") / rows ** 0.5
    sign = torch.randint(0, 2, (rows, cols), generator=g, device="cuda").to(torch.float64) * 2 - 1
    e = torch.randint(-20, 21, (rows, cols), generator=g, device="cuda", dtype=torch.int32)
    m = torch.rand(rows, cols, generator=g, dtype=torch.float64, device="cuda") + 1.0
    return sign * torch.ldexp(m, e)


def packed(X, T):
    """Grid-major dense X (K, M) -> packed-T panels of its M rows over K."""
    K, M = X.shape
    P = torch.empty(((M + T - 1) // T) * T * K, dtype=torch.float64, device="cuda")
    skgemm.pack_dev(M, K, X, 1, M, T, P)
    return P


def sample(M, N, seed, upper=False):
    rng = np.random.default_rng(seed)
    a, b = rng.integers(0, M, NS), rng.integers(0, N, NS)
    if upper:
        return np.minimum(a, b), np.maximum(a, b)
    return a, b


def host_t(X):
    """Device (K, M) -> host (M, K): state-major, so each oracle dot product
    walks contiguous memory."""
    return X.t().contiguous().cpu().numpy()


def dot2(Xt, Yt, ii, jj, K, alpha=1.0, gamma=0.0):
    """Sampled entries (ii, jj) of alpha * X^T Y + gamma from host (M, K) copies."""
    return oracle.dot2_sampled(Xt, Yt, ii, jj, alpha, gamma, x_strides=(K, 1),
                               y_strides=(1, K), K=K)


def rel(got, ref):
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


def _run_pair_ops(K, M, Xh, Yh, P16, H32, precisions, seed):
    """SYRK S = X^T X (upper) and GEMM Hs = X^T Y per precision against sampled
    Dot2; returns {precision: (err_S, err_Hs, moduli)}."""
    ii, jj = sample(M, M, seed)
    ui, uj = sample(M, M, seed + 1, upper=True)
    ref_h = dot2(Xh, Yh, ii, jj, K)
    ref_s = dot2(Xh, Xh, ui, uj, K)
    out = {}
    for prec in precisions:
        C = torch.full((M, M), np.nan, dtype=torch.float64, device="cuda")
        D = torch.full((M, M), np.nan, dtype=torch.float64, device="cuda")
        p = None if prec == NAT else prec
        oc = skgemm.dsyrk_packed_dev(K, M, P16, C, M, 1.0, 0.0, precision=p)
        od = skgemm.dgemm_packed_dev(M, M, K, P16, H32, D, M, precision=p)
        skgemm.stream_status()
        c = C.cpu().numpy()          # row j = column j of the column-major C
        d = D.cpu().numpy()
        es, eh = rel(c[uj, ui], ref_s), rel(d[ii, jj], ref_h)
        lm = (oc.slices_used_out, od.slices_used_out) if oc is not None else (0, 0)
        out[prec] = (es, eh, lm)
    return out


@pytest.mark.parametrize("K", [131073, 262144, 400000])
@pytest.mark.parametrize("M", [64, 512])
@pytest.mark.parametrize("kind", ["gauss", "stress"])
def test_long_k_gemm_syrk_all_precisions(cuda, K, M, kind):
    """GEMM and SYRK at K past one Ozaki segment (131073 = 1024 k-blocks + 1),
    at 64^3 = 262144 (config 4's largest grid) and at 4e5 (config 5's
    largest), for native FP64, Ozaki INT8 and Ozaki BF16."""
    seed = K + 7 * M + (0 if kind == "gauss" else 1)
    X = draw(kind, K, M, seed)
    Y = draw(kind, K, M, seed + 100)
    P16, H32 = packed(X, 16), packed(Y, 32)
    Xh, Yh = host_t(X), host_t(Y)
    del X, Y
    res = _run_pair_ops(K, M, Xh, Yh, P16, H32, (NAT, I8, BF), seed)
    for prec, (es, eh, lm) in res.items():
        assert es <= TOL and eh <= TOL, (prec, es, eh, lm)
    # INT8 and BF16 residues give the same integers: the same moduli are used.
    assert res[I8][2] == res[BF][2]


def test_long_k_ozaki_bf16_equals_int8_bitwise(cuda):
    """At K = 262144 the BF16 sub-segments and the INT8 segments reproduce the
    same integers, so GEMM and SYRK results are equal bit for bit."""
    K, M = 262144, 320
    X = draw("gauss", K, M, 5)
    Y = draw("gauss", K, M, 6)
    P16, H32 = packed(X, 16), packed(Y, 32)
    outs = {}
    for p in (I8, BF):
        C = torch.zeros((M, M), dtype=torch.float64, device="cuda")
        D = torch.full((M, M), np.nan, dtype=torch.float64, device="cuda")
        skgemm.dsyrk_packed_dev(K, M, P16, C, M, precision=p)
        skgemm.dgemm_packed_dev(M, M, K, P16, H32, D, M, 0.75, -0.5, precision=p)
        skgemm.stream_status()
        outs[p] = (C.cpu().numpy(), D.cpu().numpy())
    iu = np.triu_indices(M)
    assert np.array_equal(outs[I8][0][iu[1], iu[0]], outs[BF][0][iu[1], iu[0]])
    assert np.array_equal(outs[I8][1], outs[BF][1])
    Xh, Yh = host_t(X), host_t(Y)
    ii, jj = sample(M, M, 9)
    ref = dot2(Xh, Yh, ii, jj, K, 0.75, -0.5)
    assert rel(outs[BF][1][ii, jj], ref) <= TOL


@pytest.mark.parametrize("prec", [NAT, I8, BF])
def test_subspace_pair_long_k(cuda, prec):
    """S and Hs from one call (one split of Psi for both) at K = 64^3, 512
    states: equal to the separate calls bit for bit and within 1e-13 of Dot2."""
    K, M = 262144, 512
    X = draw("gauss", K, M, 11)
    Y = draw("gauss", K, M, 12)
    P16, H32 = packed(X, 16), packed(Y, 32)
    p = None if prec == NAT else prec
    S = torch.zeros((M, M), dtype=torch.float64, device="cuda")
    Hs = torch.full((M, M), np.nan, dtype=torch.float64, device="cuda")
    S1, Hs1 = torch.zeros_like(S), torch.full_like(Hs, np.nan)
    skgemm.dsubspace_packed_dev(K, M, P16, H32, S, Hs, precision=p)
    skgemm.dsyrk_packed_dev(K, M, P16, S1, M, precision=p)
    skgemm.dgemm_packed_dev(M, M, K, P16, H32, Hs1, M, precision=p)
    skgemm.stream_status()
    iu = np.triu_indices(M)
    s, s1 = S.cpu().numpy(), S1.cpu().numpy()
    assert np.array_equal(s[iu[1], iu[0]], s1[iu[1], iu[0]])
    assert torch.equal(Hs, Hs1)
    Xh, Yh = host_t(X), host_t(Y)
    ii, jj = sample(M, M, 13)
    ui, uj = sample(M, M, 14, upper=True)
    ref_h = dot2(Xh, Yh, ii, jj, K)
    ref_s = dot2(Xh, Xh, ui, uj, K)
    assert rel(Hs.cpu().numpy()[ii, jj], ref_h) <= TOL
    assert rel(s[uj, ui], ref_s) <= TOL


@pytest.mark.parametrize("nb", [1536, 2048])
@pytest.mark.parametrize("kind", ["gauss", "stress"])
def test_rotation_large_nb(cuda, nb, kind):
    """Rotations with 1536 and 2048 states (config 5's largest), native and
    Ozaki INT8, grid-packed and band-packed Psi; against sampled Dot2. The
    band-packed call equals the grid-packed one bit for bit."""
    Nd = 12288
    Psi = draw(kind, Nd, nb, nb + (0 if kind == "gauss" else 3))
    Q = draw(kind, nb, nb, nb + 50)
    Ph, Qh = Psi.cpu().numpy(), Q.cpu().numpy()
    grid = torch.empty(Nd * nb, dtype=torch.float64, device="cuda")
    skgemm.pack_dev(Nd, nb, Psi, nb, 1, 16, grid)      # grid-packed: rows = grid points
    band = packed(Psi, 16)                               # band-packed: rows = states
    rng = np.random.default_rng(nb)
    gg, bb = rng.integers(0, Nd, NS), rng.integers(0, nb, NS)
    ref = oracle.dot2_sampled(Ph, Qh, gg, bb)
    for prec in (NAT, I8):
        p = None if prec == NAT else prec
        Dg = torch.full((Nd * nb,), np.nan, dtype=torch.float64, device="cuda")
        Db = torch.full_like(Dg, np.nan)
        og = skgemm.drot_dev(Nd, nb, grid, Q, Dg, precision=p)
        ob = skgemm.drot_band_dev(Nd, nb, band, Q, Db, precision=p)
        skgemm.stream_status()
        assert torch.equal(Dg, Db)
        if og is not None:
            assert og.slices_used_out == ob.slices_used_out > 0
        got = Dg.cpu().numpy().reshape(nb // 16, Nd, 16)[bb // 16, gg, bb % 16]
        err = rel(got, ref)
        assert err <= TOL, (prec, err)


def test_rotation_bf16_refuses_nb_past_1024(cuda):
    """One FP32 accumulation over K = nb is exact only up to 1024 states: the
    BF16 rotation refuses 2048 instead of rounding."""
    Nd, nb = 64, 2048
    A = torch.zeros(Nd * nb, dtype=torch.float64, device="cuda")
    q = torch.zeros(nb * nb, dtype=torch.float64, device="cuda")
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.drot_dev(Nd, nb, A, q, torch.zeros_like(A), precision=BF)
    assert e.value.code == skgemm.ERR_UNSUPPORTED


@pytest.mark.parametrize("precision", [skgemm.PREC_NATIVE, skgemm.PREC_OZAKI_I8])
def test_kpoint_batch_with_64cubed_instance(cuda, precision):
    """A grouped launch holding a 64^3 = 262144-point instance with 1024 states
    beside smaller ones (config 4's largest grid and state count): every S
    and Hs within 1e-13 of sampled Dot2."""
    specs = [(64 ** 3, 1024), (24 ** 3, 64), (48 ** 3, 300), (32 ** 3, 777), (40 ** 3, 128)]
    items, checks, keep = [], [], []
    for i, (Ng, nb) in enumerate(specs):
        X = draw("gauss", Ng, nb, 300 + i)
        Y = draw("gauss", Ng, nb, 400 + i)
        p16, h32 = packed(X, 16), packed(Y, 32)
        S = torch.zeros(nb, nb, dtype=torch.float64, device="cuda")
        Hs = torch.full((nb, nb), np.nan, dtype=torch.float64, device="cuda")
        items += [skgemm.batch_item(skgemm.OP_SYRK_PACKED, nb, nb, Ng, p16, 0, S, nb),
                  skgemm.batch_item(skgemm.OP_GEMM_PACKED, nb, nb, Ng, p16, h32, Hs, nb)]
        checks.append((host_t(X), host_t(Y), S, Hs, Ng, nb))
        keep.append((p16, h32))  # the plan holds raw pointers into these
        del X, Y
    plan = skgemm.Plan(items, precision=precision)
    plan.run()
    plan.status()
    if precision != skgemm.PREC_NATIVE:
        assert plan.config["ozaki_problems"] == len(items)
    for i, (Xh, Yh, S, Hs, Ng, nb) in enumerate(checks):
        ii, jj = sample(nb, nb, 500 + i)
        ui, uj = sample(nb, nb, 600 + i, upper=True)
        ref_h = dot2(Xh, Yh, ii, jj, Ng)
        ref_s = dot2(Xh, Xh, ui, uj, Ng)
        assert rel(Hs.cpu().numpy()[ii, jj], ref_h) <= TOL, (Ng, nb)
        assert rel(S.cpu().numpy()[uj, ui], ref_s) <= TOL, (Ng, nb)
