"""Host logic of the batched (grouped) path, no GPU: the grouped schedule
exported by libskgemm (skgemm_batch_schedule) and a Python restatement of the
grouped kernel's segment decode (GroupSched::locate + locate_seg in
skg_fp64_kernel.cuh) checked for exact coverage: every MAC-loop iteration of
every tile of every problem is run by exactly one CTA, each tile has exactly
one owner (the CTA holding its k = 0 block), and the partials an owner waits
for are exactly the CTAs that start inside its tile."""
import bisect
import math

import numpy as np
import pytest

import skgemm

FAKE = 1 << 20  # a 16-byte aligned non-null address (never dereferenced here)


def batch_items(seed, n=40, with_empty=True):
    rng = np.random.default_rng(seed)
    items = []
    for i in range(n):
        op = int(rng.integers(0, 3))
        nb = int(np.exp(rng.uniform(np.log(16), np.log(700))))
        K = int(rng.integers(0, 3000)) if with_empty else int(rng.integers(1, 3000))
        if op == skgemm.OP_GEMM_PACKED:
            items.append(skgemm.batch_item(op, nb, int(rng.integers(1, 600)), K, FAKE, FAKE,
                                           FAKE, 600))
        elif op == skgemm.OP_SYRK_PACKED:
            items.append(skgemm.batch_item(op, nb, nb, K, FAKE, 0, FAKE, nb, 1.0, 0.5))
        else:
            nd = 16 * int(rng.integers(0, 200))
            nbr = 16 * max(1, nb // 16)
            items.append(skgemm.batch_item(op, nd, nbr, 0, FAKE, FAKE, FAKE))
    return items


def geometry(it, tile):
    """(num_tiles, iters_per_tile, tiles_n, upper) of one item, as the library
    defines them."""
    if it.op == skgemm.OP_ROT:
        M, N, K = it.M, it.N, it.N
    elif it.op == skgemm.OP_SYRK_PACKED:
        M, N, K = it.M, it.M, it.K
    else:
        M, N, K = it.M, it.N, it.K
    if M == 0 or N == 0 or K == 0:
        return 0, 0, 0, False
    tm, tn = math.ceil(M / tile), math.ceil(N / tile)
    upper = it.op == skgemm.OP_SYRK_PACKED
    nt = tn * (tn + 1) // 2 if upper else tm * tn
    return nt, math.ceil(K / 16), tn, upper


@pytest.fixture(scope="module")
def lib_loaded():
    try:
        skgemm.lib()
    except skgemm.SkgemmError as e:  # library not built
        pytest.fail(str(e))


@pytest.mark.parametrize("tile", [128, 64])
@pytest.mark.parametrize("order", [1, 2])
def test_schedule_prefix_matches_geometry(lib_loaded, tile, order):
    items = batch_items(7 + tile + order)
    perm, ib, eff = skgemm.batch_schedule(items, tile, order)
    assert sorted(perm) == list(range(len(items)))
    iters = [geometry(items[p], tile)[0] * geometry(items[p], tile)[1] for p in perm]
    assert ib[0] == 0 and all(ib[j + 1] - ib[j] == iters[j] for j in range(len(items)))
    if order == 2:
        assert all(iters[j] >= iters[j + 1] for j in range(len(iters) - 1))
    else:
        assert perm == list(range(len(items)))
    assert 0.0 < eff <= 1.0


def test_schedule_rejects_bad_items(lib_loaded):
    bad = [skgemm.batch_item(skgemm.OP_ROT, 100, 64, 0, FAKE, FAKE, FAKE)]  # Nd % 16
    with pytest.raises(skgemm.SkgemmError):
        skgemm.batch_schedule(bad, 128, 1)
    bad = [skgemm.batch_item(skgemm.OP_GEMM_PACKED, 10, 20, 5, FAKE, FAKE, FAKE, 10)]  # ldd < N
    with pytest.raises(skgemm.SkgemmError):
        skgemm.batch_schedule(bad, 128, 1)
    bad = [skgemm.batch_item(7, 10, 10, 5, FAKE, FAKE, FAKE, 10)]
    with pytest.raises(skgemm.SkgemmError):
        skgemm.batch_schedule(bad, 128, 1)
    with pytest.raises(skgemm.SkgemmError):
        skgemm.batch_schedule(batch_items(1, 3), 96, 1)


def tile_coords(t, tiles_n, upper):
    if not upper:
        return t // tiles_n, t % tiles_n
    r, rem = 0, t
    while rem >= tiles_n - r:
        rem -= tiles_n - r
        r += 1
    return r, r + rem


def decode(ib, probs, total, grid):
    """Per CTA: list of segments (pid, tile, kb, ke), following the kernel."""
    out = []
    nprob = len(probs)
    for c in range(grid):
        b, e = c * total // grid, (c + 1) * total // grid
        segs = []
        it = b
        hint = 0
        while it < e:
            # GroupSched::locate: advance from the hint by binary search.
            i = hint
            if ib[i + 1] <= it:
                i = bisect.bisect_right(ib, it, lo=i + 1, hi=nprob) - 1
            hint = i
            ipt = probs[i][1]
            local = it - ib[i]
            tile = local // ipt
            kb = local - tile * ipt
            ke = min(ipt, kb + (e - it))
            segs.append((i, tile, kb, ke))
            it += ke - kb
        out.append(segs)
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("tile,grid", [(128, 148), (64, 296), (128, 7), (64, 1)])
def test_grouped_decode_covers_every_iteration_once(lib_loaded, seed, tile, grid):
    items = batch_items(seed)
    perm, ib_all, _ = skgemm.batch_schedule(items, tile, 2)
    # The device table holds only problems with work.
    probs, ib = [], [0]
    for p in perm:
        nt, ipt, tn, up = geometry(items[p], tile)
        if nt * ipt:
            probs.append((nt, ipt, tn, up))
            ib.append(ib[-1] + nt * ipt)
    total = ib[-1]
    grid = min(grid, total)
    segs = decode(ib, probs, total, grid)
    seen = {}
    for c, ss in enumerate(segs):
        assert ss, "every CTA gets at least one iteration"
        for (pid, tile_i, kb, ke) in ss:
            assert 0 <= kb < ke <= probs[pid][1]
            for k in range(kb, ke):
                key = (pid, tile_i, k)
                assert key not in seen
                seen[key] = c
    assert len(seen) == total
    # Owners and fixups: the owner of a tile is the CTA with its k = 0 block;
    # the CTAs it waits for are the ones whose range starts inside the tile.
    for pid, (nt, ipt, tn, up) in enumerate(probs):
        for t in range(nt):
            holders = sorted({seen[(pid, t, k)] for k in range(ipt)})
            owner = seen[(pid, t, 0)]
            assert holders[0] == owner
            tile_end = ib[pid] + (t + 1) * ipt
            waited = [c2 for c2 in range(owner + 1, grid) if c2 * total // grid < tile_end]
            assert waited == holders[1:]
            tm, tn_ = tile_coords(t, tn, up)
            if up:
                assert tm <= tn_ < tn
    # Each CTA publishes at most one partial (its first segment, if it starts
    # inside a tile), so one flag per CTA suffices.
    for ss in segs:
        assert sum(1 for s in ss if s[2] != 0) <= 1
