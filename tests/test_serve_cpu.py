"""Host logic of the serving engine on its simulated executor (no GPU): the
same admission / continuous-batching scheduler as the GPU run, on a virtual
clock with a throughput model (skgemm_serve_simulate)."""
import numpy as np
import pytest

import skgemm

NATIVE, OZAKI = skgemm.PREC_NATIVE, skgemm.PREC_OZAKI_I8


def request_flop(ng, nb):
    return 5.0 * nb * nb * ng  # S nb^2 Ng + Hs 2 nb^2 Ng + rotation 2 Ng nb^2


def request_bytes(ng, nb):
    al = lambda x: (x + 511) // 512 * 512
    nb32 = (nb + 31) // 32 * 32
    return 3 * al(ng * nb * 8) + al(ng * nb32 * 8) + 3 * al(nb * nb * 8)


def test_trace_statistics():
    tr = skgemm.serve_trace(20000, rate=200.0, seed=3)
    t = np.array([x[0] for x in tr])
    ng = np.array([x[1] for x in tr])
    nb = np.array([x[2] for x in tr])
    gaps = np.diff(t)
    assert np.all(gaps >= 0)
    assert abs(gaps.mean() - 1 / 200.0) < 0.05 / 200.0          # Poisson rate
    assert abs(np.std(gaps) / gaps.mean() - 1.0) < 0.05          # exponential gaps
    assert ng.min() >= 16 and np.all(ng % 16 == 0) and np.all(nb % 16 == 0)
    assert 9000 <= ng.min() and ng.max() <= 400016
    assert 32 <= nb.min() and nb.max() <= 2048
    # log-uniform: log-sizes evenly spread between the bounds
    u = (np.log(nb) - np.log(32)) / (np.log(2048) - np.log(32))
    assert abs(np.median(u) - 0.5) < 0.03


@pytest.mark.parametrize("precision", [NATIVE, OZAKI])
@pytest.mark.parametrize("realtime", [True, False])
def test_sim_all_requests_complete_in_order(precision, realtime):
    tr = skgemm.serve_trace(3000, seed=5)
    rows, o = skgemm.serve(tr, precision=precision, simulate=True, realtime=realtime,
                           sim=(30.0, 60.0, 3000.0))
    arr = np.array([r[0] for r in rows])
    adm = np.array([r[1] for r in rows])
    done = np.array([r[2] for r in rows])
    assert np.all(adm >= arr - 1e-12) and np.all(done > adm)
    # Admission is first come, first served.
    order = np.argsort(arr, kind="stable")
    assert np.all(np.diff(adm[order]) >= -1e-12)
    assert o.peak_admitted_bytes <= 150e9
    flop = sum(request_flop(ng, nb) for _, ng, nb, _ in tr)
    assert o.flop == pytest.approx(flop, rel=1e-12)
    assert o.makespan_s == pytest.approx(done.max())
    # Every request takes at least its own work at the modelled rate.
    rate = (30.0 if precision == NATIVE else 60.0) * 1e12
    need = np.array([request_flop(ng, nb) for _, ng, nb, _ in tr]) / rate
    assert np.all(done - adm >= need * (1 - 1e-9))


def test_sim_native_is_work_conserving_offline():
    """All requests present at t = 0: the compute stream never idles while
    work is ready, so the makespan is the total work at the modelled rate
    plus the first request's input generation."""
    tr = skgemm.serve_trace(400, seed=8, nb_range=(32, 512), ng_range=(1e4, 1e5))
    rows, o = skgemm.serve(tr, simulate=True, realtime=False, sim=(30.0, 0.0, 3000.0))
    flop = sum(request_flop(ng, nb) for _, ng, nb, _ in tr)
    gen0 = max(request_bytes(ng, nb) for _, ng, nb, _ in tr) / 3000e9
    assert o.makespan_s <= flop / 30e12 + gen0 + 1e-9
    assert o.makespan_s >= flop / 30e12 * (1 - 1e-9)
    # Continuous batching: launches carry the steps of several requests.
    assert o.batches > 1 and o.mean_batch_problems > 3


def test_sim_budget_limits_admitted_data():
    tr = skgemm.serve_trace(200, seed=9)
    biggest = max(request_bytes(ng, nb) for _, ng, nb, _ in tr)
    budget = 1.5 * biggest
    rows, o = skgemm.serve(tr, simulate=True, hbm_budget=budget, realtime=False,
                           sim=(30.0, 0.0, 3000.0))
    assert o.peak_admitted_bytes <= budget
    # Tighter budget, same work: no faster than the generous one.
    rows2, o2 = skgemm.serve(tr, simulate=True, realtime=False, sim=(30.0, 0.0, 3000.0))
    assert o.makespan_s >= o2.makespan_s * (1 - 1e-9)


def test_sim_rejects_request_larger_than_budget():
    tr = [(0.0, 400000, 2048, 1)]
    with pytest.raises(skgemm.SkgemmError) as e:
        skgemm.serve(tr, simulate=True, hbm_budget=10e9)
    assert e.value.code == skgemm.ERR_OOM


def test_sim_rejects_bad_shapes():
    with pytest.raises(skgemm.SkgemmError):
        skgemm.serve([(0.0, 1000, 40, 1)], simulate=True)   # nb % 16
    with pytest.raises(skgemm.SkgemmError):
        skgemm.serve([(0.0, 1008, 4096, 1)], simulate=True, precision=OZAKI)


@pytest.mark.parametrize("precision", [NATIVE, OZAKI])
def test_sim_smallest_first_cuts_queueing(precision):
    """Aged least-work-first admission on a heavy-tailed trace (Ozaki at ~60%
    utilisation; native overloaded, demand ~1.8x its rate, as measured):
    every request completes, the same work is done, the median latency drops
    against arrival order (and, below saturation, the p99), and no request
    waits without bound (the aging discount)."""
    tr = skgemm.serve_trace(4000, rate=200.0, seed=21)
    sim = (30.0, 95.0, 900.0)
    res = {}
    for pol in (skgemm.SERVE_FIFO, skgemm.SERVE_SMALLEST):
        rows, o = skgemm.serve(tr, precision=precision, simulate=True, sim=sim, policy=pol,
                               aging_s=0.25)
        lat = np.array([d - a for a, _, d in rows])
        assert np.all(np.isfinite(lat)) and np.all(lat > 0)
        res[pol] = (np.percentile(lat, 50), np.percentile(lat, 99), lat.max(), o.flop)
    fifo, small = res[skgemm.SERVE_FIFO], res[skgemm.SERVE_SMALLEST]
    assert small[3] == fifo[3]                    # same work done
    assert small[0] < 0.5 * fifo[0]
    if precision == OZAKI:
        assert small[1] < fifo[1]
    assert small[2] < 5.0 * fifo[2] + 1.0         # the largest wait stays bounded


def test_sim_smallest_first_admits_small_request_ahead():
    """Two requests waiting behind a busy slot: the small one (arrived later)
    is admitted before the large one under SMALLEST, after it under FIFO."""
    tr = [(0.0, 400000, 2048, 1), (0.001, 400000, 2048, 2), (0.002, 16384, 64, 3)]
    order = {}
    for pol in (skgemm.SERVE_FIFO, skgemm.SERVE_SMALLEST):
        rows, _ = skgemm.serve(tr, precision=OZAKI, simulate=True, sim=(30.0, 50.0, 900.0),
                               policy=pol, ozaki_streams=1)
        order[pol] = [a for _, a, _ in rows]     # admission times
    fifo, small = order[skgemm.SERVE_FIFO], order[skgemm.SERVE_SMALLEST]
    assert fifo[2] > fifo[1]
    assert small[2] < small[1]


def test_sim_rejects_bad_policy():
    tr = skgemm.serve_trace(4, rate=200.0, seed=1)
    with pytest.raises(skgemm.SkgemmError):
        skgemm.serve(tr, precision=OZAKI, simulate=True, policy=7)
    with pytest.raises(skgemm.SkgemmError):
        skgemm.serve(tr, precision=OZAKI, simulate=True, policy=skgemm.SERVE_SMALLEST, aging_s=-1)


def test_sim_ratio_policy_bounds_the_largest_requests_wait():
    """Highest response ratio next (largest wait / work first) on the
    2000-request trace at ~93% load: all work done, median far below arrival
    order's, p99 at or below arrival order's, and the largest decile of
    requests served sooner than under aged least-work-first (which lets a
    stream of small requests hold the large ones back)."""
    tr = skgemm.serve_trace(2000, rate=200.0, seed=11)
    work = np.array([request_flop(ng, nb) for _, ng, nb, _ in tr])
    top = work >= np.percentile(work, 90)
    res = {}
    for pol in (skgemm.SERVE_FIFO, skgemm.SERVE_SMALLEST, skgemm.SERVE_RATIO):
        rows, o = skgemm.serve(tr, precision=OZAKI, simulate=True, sim=(30.0, 55.0, 3000.0),
                               policy=pol, aging_s=0.25, ozaki_streams=2)
        lat = np.array([d - a for a, _, d in rows])
        res[pol] = (np.percentile(lat, 50), np.percentile(lat, 99),
                    np.percentile(lat[top], 99), o.flop)
    fifo, small, ratio = (res[p] for p in (skgemm.SERVE_FIFO, skgemm.SERVE_SMALLEST,
                                           skgemm.SERVE_RATIO))
    assert ratio[3] == fifo[3]
    assert ratio[0] < 0.25 * fifo[0]
    assert ratio[1] <= fifo[1]
    assert ratio[2] < small[2]


def test_sim_ratio_policy_picks_the_longest_relative_wait():
    """Behind a busy slot: a small request that has waited admits before a
    large one that waited longer in absolute terms but less per unit of work."""
    tr = [(0.0, 400000, 2048, 1), (0.001, 400000, 1024, 2), (0.05, 16384, 64, 3)]
    rows, _ = skgemm.serve(tr, precision=OZAKI, simulate=True, sim=(30.0, 50.0, 900.0),
                           policy=skgemm.SERVE_RATIO, ozaki_streams=1)
    admit = [a for _, a, _ in rows]
    assert admit[2] < admit[1]
