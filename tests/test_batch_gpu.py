"""GPU parity of the batched path: grouped persistent Stream-K launches of
mixed GEMM / SYRK / rotation problems (skgemm_plan_* and skgemm_batch_dev),
called through the C ABI.

Gates: every item of a batch within relative Frobenius error 1e-13 of the
Dot2 (double-double) oracle, whatever the tile shape, problem order, grid or
graph capture; bytes outside each output's contract untouched; a replayed
graph reads the current contents of the inputs; repeated runs bitwise equal;
autotuning leaves SYRK outputs with beta != 0 as they were. Plans that run
problems through the Ozaki split (precision Ozaki or auto) meet the same
gates."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import oracle
import skgemm
from tests._cases import gaussian, uniform

pytestmark = pytest.mark.gpu
TOL = 1e-13


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64).ravel()).cuda()


class Item:
    """Host inputs, device buffers, the batch item and its oracle."""

    def __init__(self, op, seed, M, N, K, alpha=1.0, beta=0.0, ldd_pad=0):
        self.op, self.M, self.N, self.K = op, M, N, K
        self.alpha, self.beta = alpha, beta
        rng_seed = 1000 + seed
        if op == skgemm.OP_GEMM_PACKED:
            self.A = uniform((M, K), rng_seed)
            self.B = uniform((K, N), rng_seed + 1)
            self.ldd = N + ldd_pad
            self.dA = dev(oracle.pack(self.A, 16))
            self.dB = dev(oracle.pack(self.B.T, 32))
            self.D0 = np.full((M, self.ldd), 7.0)
        elif op == skgemm.OP_SYRK_PACKED:
            self.X = gaussian((K, M), rng_seed, 1.0 / np.sqrt(max(K, 1)))
            self.ldd = M + ldd_pad
            self.dA = dev(oracle.pack(self.X.T, 16))
            self.dB = None
            self.D0 = uniform((M, self.ldd), rng_seed + 2)  # column-major C: [col][row]
        else:
            self.Psi = gaussian((M, N), rng_seed, 1.0 / np.sqrt(M))
            self.Q = uniform((N, N), rng_seed + 1)
            self.ldd = 0
            self.dA = dev(oracle.grid_pack(self.Psi))
            self.dB = dev(self.Q)
            self.D0 = np.full(M * N, 7.0)
        self.dD = dev(self.D0)

    def item(self):
        return skgemm.batch_item(self.op, self.M, self.N, self.K, self.dA, self.dB, self.dD,
                                 self.ldd, self.alpha, self.beta)

    def reset(self):
        self.dD.copy_(dev(self.D0))

    def check(self, sample=0):
        """Relative Frobenius error against Dot2: over every entry, or over
        `sample` random entries (long SYRK reductions)."""
        torch.cuda.synchronize()
        out = self.dD.cpu().numpy()
        if self.M == 0 or self.N == 0:
            assert out.size == 0
            return 0.0
        if self.op == skgemm.OP_GEMM_PACKED:
            out = out.reshape(self.M, self.ldd)
            ref = oracle.dot2_matmul(self.A, self.B, self.alpha, self.beta)
            err = oracle.rel_frobenius(out[:, :self.N], ref)
            assert np.array_equal(out[:, self.N:], self.D0[:, self.N:])
        elif self.op == skgemm.OP_SYRK_PACKED and sample:
            C = out.reshape(self.M, self.ldd)
            rng = np.random.default_rng(self.M + self.K)
            a, b = rng.integers(0, self.M, sample), rng.integers(0, self.M, sample)
            i, j = np.minimum(a, b), np.maximum(a, b)
            S = oracle.dot2_sampled(self.X, self.X, i, j, x_strides=(1, self.M),
                                    y_strides=(self.M, 1), K=self.K)
            err = oracle.rel_frobenius(C[j, i], self.alpha * S + self.beta * self.D0[j, i])
            il = np.tril_indices(self.M, -1)
            assert np.array_equal(C[il[1], il[0]], self.D0[il[1], il[0]])
        elif self.op == skgemm.OP_SYRK_PACKED:
            C = out.reshape(self.M, self.ldd)  # row c = column c of C
            S = oracle.dot2_matmul(self.X.T, self.X)  # S[i, j]
            iu = np.triu_indices(self.M)       # i <= j: C[i + j*ldd] = row j, entry i
            got = C[iu[1], iu[0]]
            want = self.alpha * S[iu] + self.beta * self.D0[iu[1], iu[0]]
            err = oracle.rel_frobenius(got, want)
            il = np.tril_indices(self.M, -1)
            assert np.array_equal(C[il[1], il[0]], self.D0[il[1], il[0]])
            assert np.array_equal(C[:, self.M:], self.D0[:, self.M:])
        else:
            got = oracle.band_unpack(out.reshape(self.N // 16, self.M, 16), self.M)
            ref = oracle.dot2_matmul(self.Psi, self.Q)
            err = oracle.rel_frobenius(got, ref)
        assert err <= TOL, (self.op, self.M, self.N, self.K, err)
        return err


def mixed_batch(seed):
    G, S, R = skgemm.OP_GEMM_PACKED, skgemm.OP_SYRK_PACKED, skgemm.OP_ROT
    return [
        Item(S, seed + 0, 512, 512, 4096),
        Item(G, seed + 1, 300, 200, 1000, 1.5, 0.25, ldd_pad=3),
        Item(S, seed + 2, 100, 100, 777, 2.0, 0.5, ldd_pad=5),
        Item(R, seed + 3, 2048, 64, 0),
        Item(G, seed + 4, 17, 33, 5),
        Item(S, seed + 5, 64, 64, 13824),
        Item(G, seed + 6, 40, 50, 0, 1.0, -3.0),          # K = 0: D = gamma
        Item(S, seed + 7, 33, 33, 0, 1.0, 0.75),          # K = 0: C = beta C
        Item(R, seed + 8, 4096, 160, 0),
        Item(G, seed + 9, 257, 129, 300, -1.0, 0.0),
        Item(S, seed + 10, 1, 1, 3),
        Item(G, seed + 11, 0, 10, 10),                    # empty output
    ]


@pytest.mark.parametrize("tile", [128, 64])
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("graph", [True, False])
def test_plan_mixed_batch_matches_oracle(cuda, tile, order, graph):
    items = mixed_batch(10 * tile + order)
    plan = skgemm.Plan([it.item() for it in items], tile=tile, order=order, tune=False,
                       graph=graph)
    assert plan.config["tile"] == tile and plan.config["order"] == order
    plan.run()
    plan.status()
    for it in items:
        it.check()
    plan.close()


@pytest.mark.parametrize("grid", [1, 5, 148])
def test_plan_any_grid(cuda, grid):
    items = mixed_batch(77)
    plan = skgemm.Plan([it.item() for it in items], tile=128, order=2, grid=grid, tune=False)
    assert plan.config["grid"] == grid
    plan.run()
    plan.status()
    for it in items:
        it.check()


def test_plan_autotune_keeps_syrk_beta_outputs(cuda):
    items = mixed_batch(5)
    before = [it.dD.clone() for it in items]
    plan = skgemm.Plan([it.item() for it in items])  # tune tile and order
    cfg = plan.config
    assert cfg["candidates_timed"] == 4 and cfg["tile"] in (64, 128) and cfg["tuned_ms"] > 0
    torch.cuda.synchronize()
    for it, b in zip(items, before):
        if it.op == skgemm.OP_SYRK_PACKED and it.beta != 0.0:
            assert torch.equal(it.dD, b)
    plan.run()
    plan.status()
    for it in items:
        it.check()
    # A second plan over the same shapes reuses the tuning result.
    plan2 = skgemm.Plan([it.item() for it in items])
    assert plan2.config["candidates_timed"] == 0
    assert plan2.config["tile"] == cfg["tile"] and plan2.config["order"] == cfg["order"]


REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_plan_tuning_persists_across_processes(cuda, tmp_path):
    """A plan tuned in one process and saved (skgemm_tune_cache_save) is
    reused by a plan over the same shapes in another process after
    skgemm_tune_cache_load: no candidate is timed, the same configuration is
    chosen and the results meet the oracle. An entry that this plan's tuning
    could not have produced (Ozaki flags on a native plan) is ignored."""
    path = str(tmp_path / "tune.json")
    code = (f"import sys, json; sys.path[:0] = [{REPO!r}, "
            f"{os.path.join(REPO, 'stream-k-gemm_b200')!r}]\n"
            "import skgemm\n"
            "from tests.test_batch_gpu import mixed_batch\n"
            "items = mixed_batch(21)\n"
            "plan = skgemm.Plan([it.item() for it in items])\n"
            f"n = skgemm.tune_cache_save({path!r})\n"
            "print(json.dumps(dict(plan.config, saved=n)))\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    first = json.loads(r.stdout.strip().splitlines()[-1])
    assert first["candidates_timed"] == 4 and first["saved"] >= 1

    skgemm.tune_cache_clear()
    assert skgemm.tune_cache_load(path) == first["saved"]
    items = mixed_batch(21)
    plan = skgemm.Plan([it.item() for it in items])
    cfg = plan.config
    assert cfg["candidates_timed"] == 0
    assert (cfg["tile"], cfg["order"]) == (first["tile"], first["order"])
    plan.run()
    plan.status()
    for it in items:
        it.check()
    plan.close()

    doc = json.load(open(path))
    for e in doc["entries"]:
        e["ozaki"] = "1" * len(e["ozaki"])
    bad = tmp_path / "bad.json"
    bad.write_text('{"format": "%s", "entries": [\n' % doc["format"] +
                   ",\n".join(json.dumps(e) for e in doc["entries"]) + "\n]}\n")
    skgemm.tune_cache_clear()
    assert skgemm.tune_cache_load(bad) == len(doc["entries"])
    plan = skgemm.Plan([it.item() for it in mixed_batch(21)])
    assert plan.config["candidates_timed"] == 4 and plan.config["ozaki_problems"] == 0
    plan.close()
    skgemm.tune_cache_clear()


def test_plan_graph_replay_reads_current_inputs_and_is_deterministic(cuda):
    items = mixed_batch(9)
    plan = skgemm.Plan([it.item() for it in items], tile=128, order=2, tune=False)
    plan.run()
    plan.run()
    plan.status()
    first = [it.dD.clone() for it in items if it.op != skgemm.OP_SYRK_PACKED or it.beta == 0]
    plan.run()
    plan.status()
    again = [it.dD.clone() for it in items if it.op != skgemm.OP_SYRK_PACKED or it.beta == 0]
    assert all(torch.equal(a, b) for a, b in zip(first, again))
    # New operand values, same buffers: the replayed graph sees them.
    for it in items:
        it.reset()
        if it.op == skgemm.OP_GEMM_PACKED and it.K > 0:
            it.A = it.A * -0.5
            it.dA.copy_(dev(oracle.pack(it.A, 16)))
    torch.cuda.synchronize()
    plan.run()
    plan.status()
    for it in items:
        it.check()


def test_batch_dev_oneshot(cuda):
    items = mixed_batch(3)
    skgemm.batch_dev([it.item() for it in items])
    skgemm.stream_status()
    for it in items:
        it.check()
    # A second one-shot batch on the same stream after the first.
    for it in items:
        it.reset()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        skgemm.batch_dev([it.item() for it in items], stream=s)
        skgemm.batch_dev([it.item() for it in items if it.op != skgemm.OP_SYRK_PACKED
                          or it.beta == 0.0], stream=s)
    skgemm.stream_status(s)
    for it in items:
        if it.op == skgemm.OP_SYRK_PACKED and it.beta != 0.0:
            continue
        it.check()


def test_batch_rejects_bad_items(cuda):
    it = Item(skgemm.OP_GEMM_PACKED, 1, 10, 20, 30)
    bad = it.item()
    bad.ldd = 5
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.Plan([bad])
    assert e.value.code == skgemm.ERR_INVALID_ARG
    bad = it.item()
    bad.A = 0
    with pytest.raises(skgemm.SkgemmError):
        skgemm.batch_dev([bad])
    with pytest.raises(skgemm.SkgemmError):
        skgemm.Plan([it.item()], tile=96)


def test_batch_kpoint_set_matches_single_calls(cuda):
    """A reduced k-point set (16 instances, grids 24^3 / 32^3, states
    log-uniform in [64, 512]): each S and Hs of the grouped launch against the
    single-problem native call and, on a sample of entries, against Dot2."""
    rng = np.random.default_rng(4)
    items, singles, keep = [], [], []
    for i in range(16):
        Ng = int(rng.choice([24 ** 3, 32 ** 3]))
        nb = int(np.exp(rng.uniform(np.log(64), np.log(512))))
        g = torch.Generator(device="cuda").manual_seed(100 + i)
        Psi = torch.randn(Ng, nb, generator=g, dtype=torch.float64, device="cuda") / Ng ** 0.5
        H = torch.randn(Ng, nb, generator=g, dtype=torch.float64, device="cuda") / Ng ** 0.5
        p16 = torch.empty(((nb + 15) // 16) * 16 * Ng, dtype=torch.float64, device="cuda")
        h32 = torch.empty(((nb + 31) // 32) * 32 * Ng, dtype=torch.float64, device="cuda")
        skgemm.pack_dev(nb, Ng, Psi, 1, nb, 16, p16)
        skgemm.pack_dev(nb, Ng, H, 1, nb, 32, h32)
        S = torch.zeros(nb, nb, dtype=torch.float64, device="cuda")
        Hs = torch.zeros_like(S)
        S1, Hs1 = torch.zeros_like(S), torch.zeros_like(S)
        items += [skgemm.batch_item(skgemm.OP_SYRK_PACKED, nb, nb, Ng, p16, 0, S, nb),
                  skgemm.batch_item(skgemm.OP_GEMM_PACKED, nb, nb, Ng, p16, h32, Hs, nb)]
        skgemm.dsyrk_packed_dev(Ng, nb, p16, S1, nb)
        skgemm.dgemm_packed_dev(nb, nb, Ng, p16, h32, Hs1, nb)
        singles.append((Psi, H, S, Hs, S1, Hs1, nb))
        keep.append((p16, h32))  # the plan holds raw pointers into these
    skgemm.stream_status()
    plan = skgemm.Plan(items)
    plan.run()
    plan.status()
    for (Psi, H, S, Hs, S1, Hs1, nb) in singles:
        iu = np.triu_indices(nb)
        s, s1 = S.cpu().numpy().T, S1.cpu().numpy().T   # column-major -> [i, j]
        assert oracle.rel_frobenius(s[iu], s1[iu]) <= TOL
        assert oracle.rel_frobenius(Hs.cpu().numpy(), Hs1.cpu().numpy()) <= TOL
        P, Hh = Psi.cpu().numpy(), H.cpu().numpy()
        ii = np.random.default_rng(nb).integers(0, nb, 64)
        jj = np.random.default_rng(nb + 1).integers(0, nb, 64)
        ref = oracle.dot2_sampled(P.T, Hh, ii, jj)
        got = Hs.cpu().numpy()[ii, jj]
        assert np.max(np.abs(got - ref)) <= TOL * np.sqrt(nb) * np.abs(ref).max() + 1e-300


def ozaki_takes(it):
    """Items the Ozaki path runs: a non-empty product (rotations up to 2048 states)."""
    if it.M == 0 or it.N == 0:
        return False
    if it.op == skgemm.OP_ROT:
        return it.N <= 2048
    return it.K > 0


@pytest.mark.parametrize("graph", [True, False])
def test_plan_ozaki_precision_mixed_batch(cuda, graph):
    """Precision Ozaki: every item the split takes runs through it (K == 0 and
    empty items stay on the native path); all within 1e-13 of Dot2; a replay
    is bitwise equal to the first run."""
    items = mixed_batch(500 + int(graph))
    plan = skgemm.Plan([it.item() for it in items], tune=False, graph=graph,
                       precision=skgemm.PREC_OZAKI_I8)
    assert plan.config["ozaki_problems"] == sum(ozaki_takes(it) for it in items)
    plan.run()
    plan.status()
    for it in items:
        it.check()
    first = [it.dD.clone() for it in items]
    for it in items:
        it.reset()
    torch.cuda.synchronize()
    plan.run()
    plan.status()
    assert all(torch.equal(it.dD, f) for it, f in zip(items, first))
    plan.close()


def test_plan_ozaki_graph_reads_current_inputs(cuda):
    """The captured Ozaki kernels read the operands' current contents."""
    items = mixed_batch(640)
    plan = skgemm.Plan([it.item() for it in items], tune=False, precision=skgemm.PREC_OZAKI_I8)
    plan.run()
    plan.status()
    for it in items:
        it.reset()
        if it.op == skgemm.OP_GEMM_PACKED and it.K > 0:
            it.A = it.A * -0.5
            it.dA.copy_(dev(oracle.pack(it.A, 16)))
        elif it.op == skgemm.OP_ROT:
            it.Q = it.Q[::-1].copy()
            it.dB.copy_(dev(it.Q))
    torch.cuda.synchronize()
    plan.run()
    plan.status()
    for it in items:
        it.check()


def test_plan_auto_precision(cuda):
    """Precision auto: the cost model sends the long-reduction SYRK through the
    Ozaki split and keeps the small problems native; tuning times both
    assignments and restores SYRK outputs with beta != 0; results within
    1e-13 of Dot2 either way."""
    G, S, R = skgemm.OP_GEMM_PACKED, skgemm.OP_SYRK_PACKED, skgemm.OP_ROT
    big = Item(S, 900, 512, 512, 65536)
    small = [Item(G, 901, 64, 64, 300), Item(S, 902, 100, 100, 777, 2.0, 0.5),
             Item(R, 903, 2048, 64, 0), Item(G, 904, 40, 50, 0, 1.0, -3.0)]
    items = [big] + small
    plan = skgemm.Plan([it.item() for it in items], tune=False, precision=skgemm.PREC_AUTO)
    assert plan.config["ozaki_problems"] == 1
    plan.run()
    plan.status()
    big.check(sample=4096)
    for it in small:
        it.check()
    for it in items:
        it.reset()
    torch.cuda.synchronize()
    before = small[1].dD.clone()
    tuned = skgemm.Plan([it.item() for it in items], precision=skgemm.PREC_AUTO)
    cfg = tuned.config
    assert cfg["candidates_timed"] > 4 and cfg["ozaki_problems"] in (0, 1)
    torch.cuda.synchronize()
    assert torch.equal(small[1].dD, before)
    tuned.run()
    tuned.status()
    big.check(sample=4096)
    for it in small:
        it.check()


def test_plan_precision_options_rejected(cuda):
    it = Item(skgemm.OP_GEMM_PACKED, 1, 10, 20, 30)
    with pytest.raises(skgemm.SkgemmError):
        skgemm.Plan([it.item()], precision=7)
    with pytest.raises(skgemm.SkgemmError):
        skgemm.Plan([it.item()], precision=skgemm.PREC_OZAKI_I8, slices=5)


def test_plan_ozaki_subspace_pairs(cuda):
    """A SYRK and a GEMM of the same band-packed Psi in one Ozaki plan run as a
    subspace pair (one split of Psi): S and Hs bitwise equal to each item
    planned alone, and within 1e-13 of Dot2. An unpaired GEMM on the same Psi
    (a second H) runs on its own."""
    SY, GE = skgemm.OP_SYRK_PACKED, skgemm.OP_GEMM_PACKED
    cases, items, keep = [], [], []
    for i, (K, M) in enumerate([(4099, 100), (13824, 200), (777, 33)]):
        Psi = gaussian((K, M), 60 + i, 1.0 / np.sqrt(K))
        H = uniform((K, M), 70 + i)
        H2 = uniform((K, M), 80 + i)
        P16 = dev(oracle.pack(np.ascontiguousarray(Psi.T), 16))
        H32 = dev(oracle.pack(np.ascontiguousarray(H.T), 32))
        H32b = dev(oracle.pack(np.ascontiguousarray(H2.T), 32))
        outs = [torch.zeros(M * M, dtype=torch.float64, device="cuda") for _ in range(3)]
        its = [skgemm.batch_item(SY, M, M, K, P16, 0, outs[0], M),
               skgemm.batch_item(GE, M, M, K, P16, H32, outs[1], M, 1.5, 0.25),
               skgemm.batch_item(GE, M, M, K, P16, H32b, outs[2], M)]
        items += its
        keep.append((P16, H32, H32b))
        cases.append((Psi, H, H2, outs, its, M))
    plan = skgemm.Plan(items, tune=False, precision=skgemm.PREC_OZAKI_I8)
    assert plan.precisions() == [skgemm.PREC_OZAKI_I8] * len(items)
    plan.run()
    plan.status()
    for (Psi, H, H2, outs, its, M) in cases:
        got = [o.clone() for o in outs]
        for it, o in zip(its, outs):
            o.zero_()
            alone = skgemm.Plan([it], tune=False, graph=False, precision=skgemm.PREC_OZAKI_I8)
            alone.run()
            alone.status()
            alone.close()
        iu = np.triu_indices(M)
        s = got[0].cpu().numpy().reshape(M, M).T
        assert np.array_equal(s[iu], outs[0].cpu().numpy().reshape(M, M).T[iu])
        assert torch.equal(got[1], outs[1]) and torch.equal(got[2], outs[2])
        assert oracle.rel_frobenius(s[iu], oracle.dot2_matmul(Psi.T, Psi)[iu]) <= TOL
        assert oracle.rel_frobenius(got[1].cpu().numpy().reshape(M, M),
                                    oracle.dot2_matmul(Psi.T, H, 1.5, 0.25)) <= TOL
        assert oracle.rel_frobenius(got[2].cpu().numpy().reshape(M, M),
                                    oracle.dot2_matmul(Psi.T, H2)) <= TOL
    plan.close()


def test_plan_bf16_equals_int8(cuda):
    """A plan with BF16 residues runs the same items as the INT8 plan and
    gives the same results bit for bit (rotations with nb <= 1024)."""
    items = mixed_batch(720)
    p8 = skgemm.Plan([it.item() for it in items], tune=False, precision=skgemm.PREC_OZAKI_I8)
    p8.run()
    p8.status()
    out8 = [it.dD.clone() for it in items]
    for it in items:
        it.reset()
    torch.cuda.synchronize()
    pb = skgemm.Plan([it.item() for it in items], tune=False, precision=skgemm.PREC_OZAKI_BF16)
    assert pb.precisions().count(skgemm.PREC_OZAKI_BF16) == p8.config["ozaki_problems"]
    pb.run()
    pb.status()
    for it, o in zip(items, out8):
        assert torch.equal(it.dD, o)
        it.check()
    p8.close()
    pb.close()
