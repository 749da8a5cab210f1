"""GPU tests of the serving engine (skgemm_serve_run through the C ABI).

Each request's results are the same alone and in the mix: native FP64 within
relative Frobenius error 1e-13 (a request's grouped launch shares its
Stream-K split with whatever else is batched, so the summation order of a
tile's partials can differ), the Ozaki path bitwise (its schedule depends
only on the request's own shape). Results also match the Dot2 oracle on the
request's own inputs within 1e-13, and admission holds the HBM budget."""
import numpy as np
import pytest

import oracle
import skgemm

pytestmark = pytest.mark.gpu
TOL = 1e-13
NATIVE, OZAKI = skgemm.PREC_NATIVE, skgemm.PREC_OZAKI_I8
BUDGET = 4e9


def small_trace(n, seed, gap=0.001):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        ng = 16 * int(np.exp(rng.uniform(np.log(64), np.log(1024))))
        nb = 16 * int(rng.integers(2, 17))
        out.append((i * gap, ng, nb, 7919 * seed + i))
    return out


def buffers(ng, nb):
    nb32 = (nb + 31) // 32 * 32
    return {"S": np.zeros(nb * nb), "Hs": np.zeros(nb * nb), "Psi": np.zeros(ng * nb),
            "Psi_in": np.zeros(ng * nb), "HPsi_in": np.zeros(ng * nb32), "Q": np.zeros(nb * nb)}


def run(trace, precision, **kw):
    keep = {i: buffers(t[1], t[2]) for i, t in enumerate(trace)}
    rows, o = skgemm.serve(trace, precision=precision, hbm_budget=kw.pop("budget", BUDGET),
                           keep=keep, **kw)
    return keep, rows, o


def upper(S, nb):
    C = S.reshape(nb, nb)  # row j = column j of column-major C
    iu = np.triu_indices(nb)
    return C[iu[1], iu[0]]


def check_oracle(k, ng, nb):
    X = oracle.band_unpack(k["Psi_in"].reshape(nb // 16, ng, 16), ng)        # (Ng, nb)
    Y = _unpack32(k["HPsi_in"], ng, nb)                                     # (Ng, nb)
    Q = k["Q"].reshape(nb, nb)
    S_ref = oracle.dot2_matmul(X.T, X)
    assert oracle.rel_frobenius(upper(k["S"], nb), S_ref[np.triu_indices(nb)]) <= TOL
    assert oracle.rel_frobenius(k["Hs"].reshape(nb, nb), oracle.dot2_matmul(X.T, Y)) <= TOL
    P = oracle.band_unpack(k["Psi"].reshape(nb // 16, ng, 16), ng)
    assert oracle.rel_frobenius(P, oracle.dot2_matmul(X, Q)) <= TOL


def _unpack32(buf, ng, nb):
    """packed32 [ceil(nb/32)][Ng][32] -> (Ng, nb)."""
    nb32 = (nb + 31) // 32 * 32
    P = buf.reshape(nb32 // 32, ng, 32)
    return np.concatenate(list(P), axis=1)[:, :nb]


@pytest.mark.parametrize("precision", [NATIVE, OZAKI])
@pytest.mark.parametrize("policy", [skgemm.SERVE_FIFO, skgemm.SERVE_SMALLEST])
def test_serve_results_same_alone_and_in_mix(cuda, precision, policy):
    trace = small_trace(10, seed=1)
    mix, rows, o = run(trace, precision, realtime=False, policy=policy)
    assert o.makespan_s > 0 and o.flop > 0
    if precision == NATIVE:
        assert o.batches >= 2 and o.mean_batch_problems > 2  # requests shared launches
    for i, (t, ng, nb, sd) in enumerate(trace):
        alone, _, _ = run([(0.0, ng, nb, sd)], precision, realtime=False)
        a, m = alone[0], mix[i]
        for key in ("Psi_in", "HPsi_in", "Q"):
            assert np.array_equal(a[key], m[key])  # seeded inputs
        if precision == OZAKI:
            # S: upper triangle only (the strict lower one is not written).
            assert np.array_equal(upper(a["S"], nb), upper(m["S"], nb))
            for key in ("Hs", "Psi"):
                assert np.array_equal(a[key], m[key]), key
        else:
            assert oracle.rel_frobenius(upper(m["S"], nb), upper(a["S"], nb)) <= TOL
            assert oracle.rel_frobenius(m["Hs"], a["Hs"]) <= TOL
            assert oracle.rel_frobenius(m["Psi"], a["Psi"]) <= TOL
        if i < 4:
            check_oracle(m, ng, nb)


def test_serve_budget_holds_and_results_unchanged(cuda):
    trace = small_trace(8, seed=2)
    sizes = []
    for _, ng, nb, _ in trace:
        al = lambda x: (x + 511) // 512 * 512
        sizes.append(3 * al(ng * nb * 8) + al(ng * ((nb + 31) // 32 * 32) * 8) + 3 * al(nb * nb * 8))
    budget = 100e6 + 1.2 * max(sizes)   # the engine's fixed scratch + about one request
    tight, rows, o = run(trace, NATIVE, realtime=False, budget=budget)
    assert o.peak_admitted_bytes <= budget - o.scratch_bytes
    loose, _, _ = run(trace, NATIVE, realtime=False)
    for i, (_, ng, nb, _) in enumerate(trace):
        assert oracle.rel_frobenius(tight[i]["Psi"], loose[i]["Psi"]) <= TOL
        assert oracle.rel_frobenius(tight[i]["Hs"], loose[i]["Hs"]) <= TOL


@pytest.mark.parametrize("precision", [NATIVE, OZAKI])
def test_serve_realtime_latencies(cuda, precision):
    trace = small_trace(12, seed=3, gap=0.002)
    rows, o = skgemm.serve(trace, precision=precision, hbm_budget=BUDGET, realtime=True)
    arr = np.array([r[0] for r in rows])
    adm = np.array([r[1] for r in rows])
    done = np.array([r[2] for r in rows])
    assert np.all(adm >= arr - 1e-9) and np.all(done > adm)
    assert o.makespan_s == pytest.approx(done.max())


def test_serve_rejects_oversized_request(cuda):
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.serve([(0.0, 16000, 512, 1)], hbm_budget=200e6)
    assert e.value.code == skgemm.ERR_OOM


@pytest.mark.parametrize("precision", [NATIVE, OZAKI])
def test_serve_largest_request_matches_oracle(cuda, precision):
    """A trace holding config 5's largest request (Ng = 4e5 grid points, 2048
    states: K crosses the Ozaki path's 1023-k-block segments, the rotation
    runs with 2048 states) between small ones, under the 150 GB budget (or what
    the process has left, if less). The
    large request's S, Hs and Psi' are checked against Dot2 on sampled
    entries: 48 states (all their pairs) for S and Hs, 64 grid points x 64
    states for the rotation."""
    import torch
    big = (0.0, 400000, 2048, 99)
    trace = [(0.0, 1024, 64, 1), big, (0.0, 2048, 128, 2), (0.0, 4096, 96, 3)]
    keep = {1: buffers(big[1], big[2])}
    # The engine reserves its whole budget up front: 150 GB, or what this
    # process has left after earlier tests (the request needs about 100 GB
    # with the Ozaki path's scratch).
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    skgemm.stream_release(None)
    budget = min(150e9, torch.cuda.mem_get_info()[0] - 6e9)
    rows, o = skgemm.serve(trace, precision=precision, hbm_budget=budget, keep=keep,
                           realtime=False)
    assert o.flop > 0
    k = keep[1]
    ng, nb = big[1], big[2]
    rng = np.random.default_rng(5)
    st = np.sort(rng.choice(nb, 48, replace=False))
    P16 = k["Psi_in"].reshape(nb // 16, ng, 16)
    P32 = k["HPsi_in"].reshape(nb // 32, ng, 32)
    X = np.ascontiguousarray(P16[st // 16, :, st % 16])    # (48, Ng): states over the grid
    Y = np.ascontiguousarray(P32[st // 32, :, st % 32])
    a, b = np.meshgrid(np.arange(48), np.arange(48), indexing="ij")
    a, b = a.ravel(), b.ravel()
    ref_h = oracle.dot2_sampled(X, Y, a, b, x_strides=(ng, 1), y_strides=(1, ng), K=ng)
    Hs = k["Hs"].reshape(nb, nb)
    assert oracle.rel_frobenius(Hs[st[a], st[b]], ref_h) <= TOL
    u = a <= b
    ref_s = oracle.dot2_sampled(X, X, a[u], b[u], x_strides=(ng, 1), y_strides=(1, ng), K=ng)
    C = k["S"].reshape(nb, nb)                            # row j = column j of C
    assert oracle.rel_frobenius(C[st[b[u]], st[a[u]]], ref_s) <= TOL
    gs = np.sort(rng.choice(ng, 64, replace=False))
    R = np.ascontiguousarray(P16[:, gs, :].transpose(1, 0, 2).reshape(64, nb))  # Psi rows
    Q = k["Q"].reshape(nb, nb)
    bs = rng.integers(0, nb, 64)
    g2, b2 = np.meshgrid(np.arange(64), bs, indexing="ij")
    g2, b2 = g2.ravel(), b2.ravel()
    ref_r = oracle.dot2_sampled(R, Q, g2, b2)
    Po = k["Psi"].reshape(nb // 16, ng, 16)
    assert oracle.rel_frobenius(Po[b2 // 16, gs[g2], b2 % 16], ref_r) <= TOL
