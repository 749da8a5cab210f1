"""Benchmark of the DFT subspace step on B200 (and the reference CPU arm).

Workload (one "step"): the three subspace operations of one CheFSI iteration
on Psi = 110592 x 512 (48^3 grid points x 512 states, N(0,1)/sqrt(Nd)
entries), H*Psi an independent matrix of the same shape and distribution, and
Q = 512 x 512 U[-1,1]:
    S   = Psi^T Psi        (SYRK, upper triangle)   M(M+1)K   = 2.905e10 flop
    Hs  = Psi^T (H Psi)    (GEMM)                   2 M^2 K   = 5.798e10 flop
    Psi'= Psi Q            (rotation)               2 Nd nb^2 = 5.798e10 flop
in the reference's packed layouts (band-packed Psi for SYRK/GEMM, 32-band-
packed H*Psi, grid-packed Psi for the rotation, band-packed Psi').

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision native|ozaki|ozaki_bf16]
    python bench.py --impl reference ...     # the reference's CPU kernels

Other workloads (not the default line):
    --workload batched   64 independent SYRK+GEMM k-point instances (grid
                         points from {24^3, 32^3, 40^3, 48^3, 64^3}, states
                         log-uniform in [64, 1024]) in one tuned, graph-captured
                         grouped launch per step; --precision ozaki|auto lets the
                         plan send problems through the Ozaki split
    --workload tour      one checked launch of every auxiliary kernel (layout,
                         stencil, projector, K = 0, int8 GEMM, BF16 Ozaki, serving
                         generators, probes), untimed: the profiling driver
    --workload serving   a Poisson stream (200 requests/s) of S -> Hs -> rotate
                         requests, grid points log-uniform in [1e4, 4e5], states
                         in [32, 2048], admitted under a 150 GB HBM budget;
                         --requests sets the trace length (20000 = the full run)

Timing: K steps bracketed by a barrier and a device synchronise, CUDA events on
the launching stream, max over ranks. Every input is larger than L2 (126 MB),
so no flush is needed between steps. N > 1 runs independent replicas (the path
has no exchange step on one node): value = all ranks' flops / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "stream-k-gemm_b200"))

ND, NB = 110592, 512
ND0, NB0 = ND, NB  # the configuration's shape (set_shape changes ND, NB)
FLOP_SYRK = NB * (NB + 1) * ND
FLOP_GEMM = 2 * NB * NB * ND
FLOP_ROT = 2 * ND * NB * NB
FLOP_STEP = FLOP_SYRK + FLOP_GEMM + FLOP_ROT
METRIC = "FP64-accurate TFLOP/s (Ozaki vs native Stream-K) and p50/p99 solve latency"
WORKLOAD = "dft_subspace_step_psi110592x512"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="skgemm", choices=["skgemm", "reference"])
    ap.add_argument("--precision", default="both",
                    choices=["both", "native", "ozaki", "ozaki_bf16", "auto"],
                    help="subspace: both (default) times native and Ozaki INT8 in one run; "
                         "ozaki: INT8 residues; ozaki_bf16: BF16 residues (same results); "
                         "auto: per call (subspace) or per problem (batched), the faster path")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="subspace: requests of the serving sub-object run after the step "
                         "(native and Ozaki; 0 = skip)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nd", type=int, default=ND,
                    help="grid points (default 110592 = 48^3; smaller values for profiling)")
    ap.add_argument("--nb", type=int, default=NB, help="states (default 512)")
    ap.add_argument("--op", default="syrk",
                    choices=["syrk", "gemm", "rotation", "pair", "stencil", "halo", "nloc"],
                    help="--workload op: which call (one per step, standalone)")
    ap.add_argument("--workload", default="subspace",
                    choices=["subspace", "batched", "serving", "tour", "op"],
                    help="tour: one checked launch of every auxiliary kernel (for ncu), untimed")
    ap.add_argument("--rot-layout", default="grid", choices=["grid", "band"],
                    help="subspace: the rotation reads grid-packed Psi (the reference's "
                         "sme_gemm_trp_3d input) or the band-packed Psi of SYRK/GEMM "
                         "(skgemm_drot_band_dev, no grid-packed copy)")
    ap.add_argument("--requests", type=int, default=2000, help="serving: trace length")
    ap.add_argument("--ozaki-streams", type=int, default=2,
                    help="serving, Ozaki: requests running concurrently (each stream holds "
                         "scratch for the largest request)")
    ap.add_argument("--serve-policy", default="smallest", choices=["smallest", "fifo", "ratio"],
                    help="serving: admission order (aged least-work-first, arrival order, or "
                         "highest response ratio next)")
    ap.add_argument("--serve-aging", type=float, default=1.0,
                    help="serving, least-work-first: seconds of waiting that count as one "
                         "unit of priority")
    ap.add_argument("--instances", type=int, default=64, help="batched: k-point instances")
    ap.add_argument("--max-grid", type=int, default=0,
                    help="batched: cap on grid points per instance (smaller cases for profiling)")
    ap.add_argument("--tile", type=int, default=0, choices=[0, 64, 128],
                    help="batched: output tile (0 = autotune)")
    ap.add_argument("--no-tune", action="store_true", help="batched: cost-model plan, no timing")
    a = ap.parse_args()
    set_shape(a.nd, a.nb)
    return a


def set_shape(nd, nb):
    """Workload shape (the default is the 110592 x 512 configuration)."""
    global ND, NB, FLOP_SYRK, FLOP_GEMM, FLOP_ROT, FLOP_STEP, WORKLOAD
    ND, NB = nd, nb
    FLOP_SYRK = NB * (NB + 1) * ND
    FLOP_GEMM = 2 * NB * NB * ND
    FLOP_ROT = 2 * ND * NB * NB
    FLOP_STEP = FLOP_SYRK + FLOP_GEMM + FLOP_ROT
    WORKLOAD = f"dft_subspace_step_psi{ND}x{NB}"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = self.smi_id(gpu_index)
        self.proc = None
        self.path = None

    @staticmethod
    def smi_id(index: int) -> str:
        """nvidia-smi's id of CUDA device `index`: its PCI bus id, which stays
        right when CUDA_VISIBLE_DEVICES remaps the ordinals."""
        try:
            import torch
            pr = torch.cuda.get_device_properties(index)
            return f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        except Exception:
            return str(index)

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[4:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        peak = max(r[0] for r in rows)
        load = [r for r in rows if r[0] >= 0.5 * peak] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i in range(4)
                          if r[2][i + 1].lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in load),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------------ distributed
def dist_setup(n, backend="nccl"):
    """One process per GPU (torchrun env): (rank, world, torch.distributed or
    None). The replicas exchange only their timings; `backend` "gloo" runs
    the same plumbing on CPU (tests)."""
    import torch
    if n <= 1 or "RANK" not in os.environ:
        return 0, 1, None
    import datetime
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", 0))
    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist.get_rank(), dist.get_world_size(), dist


def max_over_ranks(x, dist):
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    import torch
    if dist is not None:
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def job_throughput(flop_per_step, steps, world, max_ms):
    """Whole-job TFLOP/s of `world` replicas that each ran `steps` steps,
    timed as the maximum over ranks (weak scaling)."""
    return flop_per_step * steps * world / (max_ms * 1e-3) / 1e12


# ------------------------------------------------------------------ inputs
N_CHECK_STATES = 48    # states whose pairs sample S and Hs for the in-run error
N_CHECK_ROWS = 64      # grid rows sampling the rotation's error
FALLBACK_HBM_GBS = 6650.0


def make_inputs(device):
    """Seeded synthetic inputs of the workload, generated on the device; also
    the slices the in-run accuracy check needs (columns of Psi and H Psi for
    N_CHECK_STATES states, N_CHECK_ROWS rows of Psi)."""
    import torch
    import skgemm
    g = torch.Generator(device=device).manual_seed(20240611)
    scale = 1.0 / ND ** 0.5
    psi = torch.randn(ND, NB, generator=g, dtype=torch.float64, device=device) * scale
    hpsi = torch.randn(ND, NB, generator=g, dtype=torch.float64, device=device) * scale
    q = torch.rand(NB, NB, generator=g, dtype=torch.float64, device=device) * 2 - 1
    band = torch.empty(ND * NB, dtype=torch.float64, device=device)
    h32 = torch.empty_like(band)
    grid = torch.empty_like(band)
    skgemm.pack_dev(NB, ND, psi, 1, NB, 16, band)   # band-packed Psi
    skgemm.pack_dev(NB, ND, hpsi, 1, NB, 32, h32)   # 32-band-packed H Psi
    skgemm.pack_dev(ND, NB, psi, NB, 1, 16, grid)   # grid-packed Psi
    gc = torch.Generator().manual_seed(7)
    st = torch.randperm(NB, generator=gc)[:min(N_CHECK_STATES, NB)].sort().values
    gs = torch.randperm(ND, generator=gc)[:min(N_CHECK_ROWS, ND)].sort().values
    check = {"st": st, "gs": gs, "psi_cols": psi[:, st.to(device)].contiguous(),
             "hpsi_cols": hpsi[:, st.to(device)].contiguous(),
             "psi_rows": psi[gs.to(device)].contiguous()}
    torch.cuda.synchronize()
    del psi, hpsi
    return band, h32, grid, q, check


def dd_products(X, Y, chunk=8192):
    """X^T Y for X (K, m), Y (K, n) on the device in double-double arithmetic:
    Dekker's exact products (each factor split into 26-bit halves) and
    Knuth's TwoSum in a pairwise tree, the error terms carried beside the sums;
    every step is a separate elementwise torch operation, so nothing is fused
    into an FMA. Accurate to about 2^-104 of sum |x y|: an independent
    reference for the library's results (it uses none of the library's
    kernels)."""
    import torch
    c = 134217729.0  # 2^27 + 1

    def split(a):
        t = a * c
        hi = t - (t - a)
        return hi, a - hi

    def two_sum(a, b):
        s = a + b
        bb = s - a
        return s, (a - (s - bb)) + (b - bb)

    m, n = X.shape[1], Y.shape[1]
    hi_tot = torch.zeros(m, n, dtype=torch.float64, device=X.device)
    lo_tot = torch.zeros_like(hi_tot)
    for k0 in range(0, X.shape[0], chunk):
        x = X[k0:k0 + chunk, :, None]
        y = Y[k0:k0 + chunk, None, :]
        p = x * y
        xh, xl = split(x)
        yh, yl = split(y)
        e = ((xh * yh - p) + xh * yl + xl * yh) + xl * yl    # p + e = x y exactly
        while p.shape[0] > 1:
            if p.shape[0] % 2:
                p = torch.cat([p, torch.zeros_like(p[:1])])
                e = torch.cat([e, torch.zeros_like(e[:1])])
            s, err = two_sum(p[0::2], p[1::2])
            e = e[0::2] + e[1::2] + err
            p = s
        hi_tot, err = two_sum(hi_tot, p[0])
        lo_tot = lo_tot + e[0] + err
    return hi_tot + lo_tot


def subspace_errors(S, Hs, Pn, check):
    """Relative Frobenius errors of S (upper triangle), Hs and Psi' on the
    sampled entries against the double-double reference."""
    import torch
    st, gs = check["st"], check["gs"]
    X, Y, R = check["psi_cols"], check["hpsi_cols"], check["psi_rows"]
    dev = X.device
    s_ref = dd_products(X, X)
    h_ref = dd_products(X, Y)
    q = check["q"]
    r_ref = dd_products(R.t().contiguous(), q)            # (rows, NB)
    sd, gd = st.to(dev), gs.to(dev)
    a, b = torch.meshgrid(torch.arange(len(st), device=dev), torch.arange(len(st), device=dev),
                          indexing="ij")
    up = a <= b
    # S is column-major: S[i + j*NB] = S(i, j), i <= j.
    s_got = S.view(-1)[(sd[a] + sd[b] * NB)[up]]
    h_got = Hs.view(-1)[sd[a] * NB + sd[b]].view(len(st), len(st))
    bb = torch.arange(NB, device=dev)
    P = Pn.view(NB // 16, ND, 16)
    r_got = P[(bb // 16)[None, :], gd[:, None], (bb % 16)[None, :]]

    def rel(x, r):
        return float(torch.linalg.norm(x - r) / torch.linalg.norm(r))

    return {"S": rel(s_got, s_ref[up]), "Hs": rel(h_got, h_ref), "Psi_Q": rel(r_got, r_ref)}


def measured_peaks():
    """HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json when present, else
    the pool's fallback figure; returns (value, source)."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth)"
    except (OSError, KeyError, ValueError, TypeError):
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"


# ----------------------------------------------------------- GPU arm
PREC_NAMES = ("native", "ozaki", "ozaki_bf16", "auto")


def _prec(skgemm, name):
    return {"native": None, "ozaki": skgemm.PREC_OZAKI_I8,
            "ozaki_bf16": skgemm.PREC_OZAKI_BF16, "auto": skgemm.PREC_AUTO}[name]


class Step:
    """One subspace step (S, Hs, Psi') on device-resident inputs."""

    def __init__(self, skgemm, prec, band, h32, grid, q, S, Hs, Pn, stream, rot_layout):
        self.k, self.prec = skgemm, prec
        self.band, self.h32, self.grid, self.q = band, h32, grid, q
        self.S, self.Hs, self.Pn, self.stream = S, Hs, Pn, stream
        self.rot_layout = rot_layout
        self.opts = {}

    def __call__(self, evs=None):
        k, s = self.k, self.stream
        if evs:
            evs[0].record(s)
        if self.prec is None:
            k.dsyrk_packed_dev(ND, NB, self.band, self.S, NB, 1.0, 0.0, stream=s)
            if evs:
                evs[1].record(s)
            k.dgemm_packed_dev(NB, NB, ND, self.band, self.h32, self.Hs, NB, 1.0, 0.0, stream=s)
        else:
            # S and Hs share one split of Psi (skgemm_dsubspace_packed_dev).
            self.opts["pair"] = k.dsubspace_packed_dev(ND, NB, self.band, self.h32, self.S,
                                                       self.Hs, stream=s, precision=self.prec)
            if evs:
                evs[1].record(s)
        if evs:
            evs[2].record(s)
        if self.rot_layout == "band":
            o = k.drot_band_dev(ND, NB, self.band, self.q, self.Pn, stream=s, precision=self.prec)
        else:
            o = k.drot_dev(ND, NB, self.grid, self.q, self.Pn, stream=s, precision=self.prec)
        self.opts["rot"] = o
        if evs:
            evs[3].record(s)


def time_step(step, args, dist, torch):
    """W untimed steps, then K steps bracketed by barriers and a device
    synchronise, CUDA events on the launching stream; clocks sampled during
    the timed region. Returns (max-over-ranks total ms, per-op ms array,
    clocks)."""
    import numpy as np
    stream = step.stream
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    for _ in range(args.warmup):
        step()
    step.k.stream_status(stream)
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(dist)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(args.steps):
        step(ev[i])
    t1.record(stream)
    barrier(dist)
    clk = clocks.stop()
    step.k.stream_status(stream)
    total_ms = max_over_ranks(t0.elapsed_time(t1), dist)
    per_op = np.array([[ev[i][j].elapsed_time(ev[i][j + 1]) for j in range(3)]
                       for i in range(args.steps)])
    return total_ms, per_op, clk


def time_calls(fn, stream, torch, reps=10, warm=2):
    """Mean ms of fn() over reps calls (CUDA events on `stream`)."""
    for _ in range(warm):
        fn()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / reps


def _timed_kernels(skgemm, fn, stream, steps):
    """{kernel: (launches, total ms)} of `steps` calls of fn() with the
    library's event timer on."""
    skgemm.kernel_timing(True)
    for _ in range(steps):
        fn()
    skgemm.stream_status(stream)
    rep = skgemm.kernel_timing_report()
    skgemm.kernel_timing(False)
    return rep


def kernel_rooflines(skgemm, step, torch, steps, peaks, band, grid, q, S, Pn):
    """Per-kernel figures of this precision, measured with the library's
    event timer outside the timed region.

    `share` / `ms_in_step`: from `steps` more subspace steps (in the Ozaki
    pair, H Psi's norms and conversion run on a helper stream beside Psi's,
    so two kernels can share the GPU there). `achieved` / `frac`: from a
    serial pass of standalone calls (SYRK, then the rotation, one stream,
    one kernel at a time), each kernel rated against its roofline: FP64
    Stream-K kernels against the FP64 DMMA peak, INT8 products against the
    INT8 peak, conversions / norms / the rotation's reconstruction against
    HBM. Algorithmic work per launch: SYRK M (M+1) K, rotation 2 Nd nb^2
    flop (INT8 ops: the same times the moduli count L); a conversion 8 + L
    bytes per element (8 + 2 L for BF16 residues; the SYRK's operand by
    convert_tma_kernel after a norm pass of 8 bytes per element, the
    rotation's in one pass by convert_short_kernel), the rotation's
    reconstruction L + 8 bytes per element (element = one of the Nd x nb
    operand's)."""
    fp64_peak, i8_peak, hbm = peaks
    rep = _timed_kernels(skgemm, step, step.stream, steps)
    total = sum(ms for _, ms in rep.values()) or 1.0
    out = {name: {"launches_per_step": round(n / steps, 2),
                  "ms_in_step": round(ms / n, 4), "share": round(ms / total, 4)}
           for name, (n, ms) in sorted(rep.items(), key=lambda kv: -kv[1][1])}
    E = ND * NB
    s = step.stream
    opts = {}

    def serial():
        opts["syrk"] = skgemm.dsyrk_packed_dev(ND, NB, band, S, NB, stream=s, precision=step.prec)
        opts["rot"] = skgemm.drot_dev(ND, NB, grid, q, Pn, stream=s, precision=step.prec)

    alone = _timed_kernels(skgemm, serial, s, steps)
    if step.prec is None:
        work = {"fp64_streamk_kernel64": (FLOP_SYRK + FLOP_ROT, "TFLOP/s", fp64_peak, "tensor")}
    else:
        Ls, Lr = opts["syrk"].slices_used_out, opts["rot"].slices_used_out
        rb = 2 if step.prec == skgemm.PREC_OZAKI_BF16 else 1
        work = {"i8_gemm_kernel": (Ls * FLOP_SYRK, "TOP/s", i8_peak, "tensor"),
                "i8_gemm2_kernel": (Ls * FLOP_SYRK, "TOP/s", i8_peak, "tensor"),
                "i8_rot_kernel": (Lr * FLOP_ROT, "TOP/s", i8_peak, "tensor"),
                "convert_tma_kernel": (E * (8 + rb * Ls), "GB/s", hbm, "hbm"),
                "norm_partials_kernel": (E * 8, "GB/s", hbm, "hbm"),
                "convert_short_kernel": (E * (8 + rb * Lr), "GB/s", hbm, "hbm"),
                "crt_residues_band_kernel": (E * (rb * Lr + 8), "GB/s", hbm, "hbm")}
    if step.prec is None:
        # the GEMM's kernel from the step itself (one launch per step, serial)
        n, ms = rep.get("fp64_streamk_kernel", (0, 0.0))
        if n:
            ach = FLOP_GEMM * n / (ms * 1e-3) / 1e12
            out["fp64_streamk_kernel"].update({
                "bound": "tensor", "ms_alone": round(ms / n, 4), "achieved": round(ach, 3),
                "peak": round(fp64_peak, 3), "unit": "TFLOP/s", "frac": round(ach / fp64_peak, 4)})
    for name, (n, ms) in alone.items():
        row = out.setdefault(name, {"launches_per_step": 0, "ms_in_step": None, "share": 0.0})
        row["ms_alone"] = round(ms / n, 4)
        if name in work:
            w, unit, peak, bound = work[name]
            scale = 1e12 if unit in ("TFLOP/s", "TOP/s") else 1e9
            ach = w * steps / (ms * 1e-3) / scale
            row.update({"bound": bound, "achieved": round(ach, 3), "peak": round(peak, 3),
                        "unit": unit, "frac": round(ach / peak, 4)})
    return out


def run_gpu(args):
    import numpy as np
    import torch
    import skgemm

    rank, world, dist = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    names = ["native", "ozaki"] if args.precision == "both" else [args.precision]
    band, h32, grid, q, check = make_inputs(dev)
    check["q"] = q
    S = torch.zeros(NB, NB, dtype=torch.float64, device=dev)
    Hs = torch.zeros_like(S)
    Pn = torch.empty_like(band)
    stream = torch.cuda.current_stream()
    fp64_peak = skgemm.probe_fp64_peak()
    i8_peak = skgemm.probe_i8_peak()
    hbm, hbm_src = measured_peaks()

    res = {}
    for name in names:
        step = Step(skgemm, _prec(skgemm, name), band, h32, grid, q, S, Hs, Pn, stream,
                    args.rot_layout)
        total_ms, per_op, clk = time_step(step, args, dist, torch)
        step_ms = per_op.sum(axis=1)
        r = {"tflops": round(job_throughput(FLOP_STEP, args.steps, world, total_ms), 3),
             "ms_per_step": round(total_ms / args.steps, 4),
             "latency_ms": {"p50": round(float(np.percentile(step_ms, 50)), 4),
                            "p99": round(float(np.percentile(step_ms, 99)), 4)},
             "clocks": clk}
        if step.prec is None:
            ops = {"syrk": (per_op[:, 0], FLOP_SYRK), "gemm": (per_op[:, 1], FLOP_GEMM),
                   "rotation": (per_op[:, 2], FLOP_ROT)}
        else:
            ops = {"syrk+gemm": (per_op[:, 0] + per_op[:, 1], FLOP_SYRK + FLOP_GEMM),
                   "rotation": (per_op[:, 2], FLOP_ROT)}
        r["op_ms"] = {k: round(float(v.mean()), 4) for k, (v, _) in ops.items()}
        r["op_tflops"] = {k: round(f / v.mean() / 1e9, 3) for k, (v, f) in ops.items()}
        if step.prec is not None:
            r["moduli"] = {"syrk+gemm": step.opts["pair"].slices_used_out,
                           "rotation": step.opts["rot"].slices_used_out}
        # Accuracy of this precision's results (the last timed step's outputs).
        r["rel_frobenius_error"] = {k: float(f"{v:.3e}")
                                    for k, v in subspace_errors(S, Hs, Pn, check).items()}
        r["kernels"] = kernel_rooflines(skgemm, step, torch, 3, (fp64_peak, i8_peak, hbm),
                                        band, grid, q, S, Pn)
        res[name] = r

    # Standalone SYRK and GEMM (the reference's one-call-at-a-time use).
    alone = {}
    if len(names) > 1 or names[0] != "native":
        for name in names:
            p = _prec(skgemm, name)
            alone[name] = {
                "syrk_ms": round(time_calls(lambda: skgemm.dsyrk_packed_dev(
                    ND, NB, band, S, NB, stream=stream, precision=p), stream, torch), 4),
                "gemm_ms": round(time_calls(lambda: skgemm.dgemm_packed_dev(
                    NB, NB, ND, band, h32, Hs, NB, stream=stream, precision=p), stream, torch), 4),
                "rotation_ms": round(time_calls(lambda: skgemm.drot_dev(
                    ND, NB, grid, q, Pn, stream=stream, precision=p), stream, torch), 4)}
        skgemm.stream_status(stream)

    ok = {n: max(r["rel_frobenius_error"].values()) <= 1e-13 for n, r in res.items()}
    head = "ozaki" if "ozaki" in res and ok["ozaki"] else names[0]
    H = res[head]
    per_kernel = H["kernels"]
    dom = max(per_kernel, key=lambda k: per_kernel[k]["share"])
    dk = per_kernel[dom]
    traffic = read_profile_traffic(dom)
    line = {
        "metric": METRIC, "value": H["tflops"], "unit": "TFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": H["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "Nd": ND, "nb": NB, "ops": ["syrk", "gemm", "rotation"],
                   "precision": head,
                   "value_is": (f"the {head} step (FP64-accurate: measured error <= 1e-13 on "
                                f"every result)" if ok[head] else
                                f"the {head} step (measured error above 1e-13)"),
                   "rot_layout": args.rot_layout, "parallelism": f"replicas{world}",
                   "flop_per_step": FLOP_STEP, "l2": "inputs larger than L2 (453 MB each)"},
        "latency_ms": H["latency_ms"],
        "roofline": {"bound": dk.get("bound"), "achieved": dk.get("achieved"),
                     "peak": dk.get("peak"), "unit": dk.get("unit"), "frac": dk.get("frac"),
                     "traffic": traffic, "kernel": dom, "share_of_step": dk["share"],
                     "peak_source": {"tensor": "measured in this run (skgemm_probe_fp64_peak / "
                                               "skgemm_probe_i8_peak)",
                                     "hbm": hbm_src}.get(dk.get("bound"), None),
                     "timing": "CUDA events around each launch on its stream (library kernel "
                               "timer), standalone SYRK + rotation calls after the timed "
                               "region; share = of the step's kernel time"},
        "clocks": H["clocks"],
        "gpu_launches": 0,
    }
    line["native"] = res.get("native")
    line["ozaki"] = res.get("ozaki")
    if args.precision not in ("both", "native", "ozaki"):
        line[args.precision] = res[args.precision]
    # Every kernel of the library in a step, counted by its event timer.
    line["gpu_launches"] = int(round(sum(k["launches_per_step"] for k in per_kernel.values())
                                     * args.steps))
    if alone:
        line["standalone_ms"] = alone
        if "native" in alone and "ozaki" in alone:
            a, o = alone["native"], alone["ozaki"]
            line["speedup_ozaki_vs_native"] = {
                "step": round(res["native"]["ms_per_step"] / res["ozaki"]["ms_per_step"], 3),
                "syrk": round(a["syrk_ms"] / o["syrk_ms"], 3),
                "gemm": round(a["gemm_ms"] / o["gemm_ms"], 3),
                "rotation": round(a["rotation_ms"] / o["rotation_ms"], 3)}
    del check
    if not args.no_e2e:
        line["e2e"] = run_e2e(args, band, h32, grid, q, dist, _prec(skgemm, head), head)
    del band, h32, grid, S, Hs, Pn
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    skgemm.stream_release(stream)
    if world == 1 and args.serve_requests > 0:
        # Both precisions under the default admission policy and, on the same
        # box, under arrival order (FIFO) for comparison.
        line["serving"] = {}
        for n in ("native", "ozaki"):
            for pol in (args.serve_policy, "fifo"):
                key = n if pol == args.serve_policy else f"{n}_fifo"
                if key in line["serving"]:
                    continue
                try:
                    line["serving"][key] = serve_measure(args, n, args.serve_requests, rank,
                                                         None, pol)
                except skgemm.SkgemmError as e:  # keep the step's line; say what failed
                    line["serving"][key] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def read_profile_traffic(kernel):
    """DRAM bytes (read + write) per launch of `kernel` on this workload, from
    the committed ncu summaries (their `traffic_bytes_per_launch <kernel>:`
    lines), or None."""
    pdir = os.path.join(REPO, "profiles")
    if not os.path.isdir(pdir):
        return None
    key = f"traffic_bytes_per_launch {kernel}:"
    for fn in sorted(os.listdir(pdir)):
        for line in open(os.path.join(pdir, fn)):
            if line.startswith(key):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


def run_e2e(args, band, h32, grid, q, dist, prec, name):
    """Same step through the blocking host-pointer C ABI (the reference-facing
    calls, with the precision selector of their `_opt` forms): inputs copied
    from pinned host memory and results read back every step."""
    import torch
    import skgemm
    hb = band.cpu().pin_memory().numpy()
    hh = h32.cpu().pin_memory().numpy()
    hg = grid.cpu().pin_memory().numpy()
    hq = q.cpu().pin_memory().numpy().ravel()
    S = torch.zeros(NB * NB, dtype=torch.float64).pin_memory().numpy()
    Hs = torch.zeros(NB * NB, dtype=torch.float64).pin_memory().numpy()
    Pn = torch.zeros(ND * NB, dtype=torch.float64).pin_memory().numpy()

    def step():
        skgemm.sme_syrk.compute(ND, NB, hb, S, 1.0, 0.0, precision=prec)
        skgemm.gemm.compute_packed(NB, NB, ND, hb, hh, Hs, 1.0, 0.0, precision=prec)
        skgemm.sme_gemm_trp_3d.compute(ND, NB, hg, hq, Pn, precision=prec)

    steps = max(2, min(args.steps, 5))
    for _ in range(2):
        step()
    barrier(dist)
    t = time.perf_counter()
    for _ in range(steps):
        step()
    el = max_over_ranks(time.perf_counter() - t, dist)
    h2d = hb.nbytes * 2 + hh.nbytes + hg.nbytes + hq.nbytes + S.nbytes
    d2h = S.nbytes + Hs.nbytes + Pn.nbytes
    world = 1 if dist is None else dist.get_world_size()
    api = ("skgemm_dsyrk_packed + skgemm_dgemm_packed + skgemm_drot (host pointers)"
           if prec is None else
           "skgemm_dsyrk_packed_opt + skgemm_dgemm_packed_opt + skgemm_drot_opt (host pointers, "
           f"precision {name})")
    return {"value": round(FLOP_STEP * steps * world / el / 1e12, 4), "unit": "TFLOP/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": round(el / steps * 1e3, 3), "steps": steps, "precision": name,
            "api": api}


# ------------------------------------------------------------ one op
def run_op(args):
    """One standalone call per step (the reference's one-call-at-a-time use)
    on the subspace shapes: SYRK S = Psi^T Psi, GEMM Hs = Psi^T H Psi, the
    rotation Psi Q, or the S + Hs pair (one line per precision, two with
    --precision both); or the H Psi producer on the same Psi: the periodic
    halo, the stencil, the nonlocal projector. For profiling a single op and
    timing it alone. Prints {"op", "precision", "ms", ...}."""
    import numpy as np
    import torch
    import skgemm
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    band, h32, grid, q, _ = make_inputs(dev)
    S = torch.zeros(NB * NB, dtype=torch.float64, device=dev)
    Hs = torch.zeros_like(S)
    Pn = torch.empty_like(band)
    s = torch.cuda.current_stream()
    if args.op == "nloc":
        # The nonlocal projector H Psi += V_nloc Psi on the same Psi (48^3
        # grid points, 512 bands): 64 atoms x 2 periodic images, 800 random
        # grid rows x 16 columns per projector (seeded).
        rng = np.random.default_rng(8)
        atoms, images, nrow, ncol = 64, 2, 800, 16
        nproj = atoms * images
        proj = skgemm.NlocProjector(
            np.full(nproj, nrow), np.full(nproj, ncol),
            np.repeat(np.arange(1, atoms + 1), images),
            np.append(np.repeat(np.arange(atoms) * ncol, images), atoms * ncol),
            np.concatenate([rng.permutation(ND)[:nrow] for _ in range(nproj)]),
            rng.uniform(-1, 1, nproj * nrow * ncol), rng.uniform(-0.5, 0.5, nproj * ncol), ND)
        hpsi = torch.zeros_like(band)
        fn = lambda: proj.apply(NB, 0.01, band, hpsi, 32, stream=s)
        ms = time_calls(fn, s, torch, reps=max(1, args.steps), warm=max(0, args.warmup))
        rep = _timed_kernels(skgemm, fn, s, max(1, args.steps))
        skgemm.stream_status(s)
        proj.close()
        flop = 2 * 2 * nproj * nrow * ncol * NB
        print(json.dumps({"workload": f"op_nloc_48cubed_x{NB}_64atoms_x2", "op": "nloc",
                          "precision": "f64", "ms": round(ms, 4),
                          "tflops": round(flop / ms / 1e9, 3),
                          "kernels_ms": {k: round(v[1] / v[0], 4) for k, v in rep.items()}}),
              flush=True)
        return
    if args.op in ("stencil", "halo"):
        # The H Psi producer on the same Psi (48^3 = 110592 grid points, 512
        # bands): the periodic halo (band-packed Psi -> extended) or the
        # 6th-order stencil (extended -> 32-band-packed H Psi), alone.
        n = 48
        ext = torch.empty((NB + 15) // 16 * (n + 12) ** 3 * 16, dtype=torch.float64, device=dev)
        a_diag = torch.rand(ND, dtype=torch.float64, device=dev)
        cx = [0.0, -1.0 / 12, 2.0 / 3, -2.5, 8.0 / 3, -1.0 / 4, 1.0 / 30]
        hpsi = torch.empty_like(band)
        skgemm.halo_periodic_dev(n, n, n, NB, band, ext, stream=s)
        if args.op == "halo":
            fn = lambda: skgemm.halo_periodic_dev(n, n, n, NB, band, ext, stream=s)
            nbytes = band.numel() * 8 + ext.numel() * 8
        else:
            fn = lambda: skgemm.stencil_ext_dev(n, n, n, NB, ext, a_diag, cx, cx, cx, -0.5, hpsi,
                                                32, stream=s)
            nbytes = ext.numel() * 8 + a_diag.numel() * 8 + hpsi.numel() * 8
        ms = time_calls(fn, s, torch, reps=max(1, args.steps), warm=max(0, args.warmup))
        skgemm.stream_status(s)
        hbm, src = measured_peaks()
        gbs = nbytes / ms / 1e6
        print(json.dumps({"workload": f"op_{args.op}_hpsi_48cubed_x{NB}", "op": args.op,
                          "precision": "f64", "ms": round(ms, 4),
                          "algorithmic_bytes": int(nbytes), "gbs": round(gbs, 1),
                          "frac_of_hbm": round(gbs / hbm, 4), "hbm_peak_source": src}),
              flush=True)
        return
    for name in (["native", "ozaki"] if args.precision == "both" else [args.precision]):
        p = _prec(skgemm, name)
        calls = {
            "syrk": (lambda: skgemm.dsyrk_packed_dev(ND, NB, band, S, NB, stream=s, precision=p),
                     FLOP_SYRK),
            "gemm": (lambda: skgemm.dgemm_packed_dev(NB, NB, ND, band, h32, Hs, NB, stream=s,
                                                     precision=p), FLOP_GEMM),
            "rotation": (lambda: skgemm.drot_dev(ND, NB, grid, q, Pn, stream=s, precision=p),
                         FLOP_ROT),
            "pair": (lambda: skgemm.dsubspace_packed_dev(ND, NB, band, h32, S, Hs, stream=s,
                                                         precision=p), FLOP_SYRK + FLOP_GEMM)}
        fn, flop = calls[args.op]
        ms = time_calls(fn, s, torch, reps=max(1, args.steps), warm=max(0, args.warmup))
        rep = _timed_kernels(skgemm, fn, s, max(1, args.steps))  # a separate pass, timer on
        skgemm.stream_status(s)
        print(json.dumps({"workload": f"op_{args.op}_{WORKLOAD}", "op": args.op,
                          "precision": name, "ms": round(ms, 4),
                          "tflops": round(flop / ms / 1e9, 3),
                          "kernels_ms": {k: round(v[1] / v[0], 4) for k, v in rep.items()}}),
              flush=True)


# ------------------------------------------------------------ kernel tour
def run_tour(args=None) -> None:
    """One launch of every auxiliary kernel of the library on a representative
    workload, for profiling (ncu) and as a quick end-to-end exercise; every
    result is checked for a device-side error, nothing is timed:

      pack_kernel<16>, pack_kernel<32>   dense 110592 x 512 -> band-packed (453 MB)
      band_grid_kernel (both ways)       110592 x 512 band <-> grid packed (453 MB)
      unpack_kernel<16>                  grid-packed -> column-major (linalg_unpack_c16)
      fp64_streamk_kernel_ak             the rotation on band-packed Psi, 8192 x 1024
                                         (512 tiles of 128 x 128: the 128-row kernel)
      fp64_streamk_kernel64_ak,          the rotation on band-packed Psi, 110592 x 512,
      convert_short_kernel (KM)          native and Ozaki (K-major operand reads)
      halo_periodic_kernel,              H Psi on the 48^3 grid (= 110592 points) x 512:
      stencil_staged_kernel<32>          periodic halo, then the 6th-order stencil
      nloc_forward / nloc_chi_c /        the nonlocal projector on the same Psi: 64 atoms
      nloc_backward<32>                  x 2 periodic images, 800 rows x 16 columns each
      k0_kernel                          GEMM with K = 0 (D = gamma), 4096 x 4096, through
                                         the regular and the allocation-free entries
      sum_parts_kernel                   the host GEMM's k-chunk combine, 2048 x 2048 x 32768
      i8_gemm_kernel + sum_partials      the public exact int8 GEMM, 4096 x 4096 x 4096
      BF16 Ozaki kernels                 GEMM 512 x 512 x 110592, rotation 110592 x 512
      gen_normal / gen_uniform           a two-request serving trace (inputs made on
                                         the device from seeds)
      dmma_peak_kernel, i8_peak_kernel   the peak probes
    """
    import numpy as np
    import torch
    import skgemm

    np.seterr(all="ignore")
    assert torch.cuda.is_available(), "the kernel tour needs a GPU"
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = torch.Generator(device=dev).manual_seed(5)

    # The rotation's 128 x 128 K-major kernel (fewer than 4 tiles per SM),
    # first, while little memory is held: Psi 67 MB, Q 8 MB.
    nd, nb = 8192, 1024
    psi = torch.randn(nd * nb, generator=g, dtype=torch.float64, device=dev) / nd ** 0.5
    q = torch.rand(nb * nb, generator=g, dtype=torch.float64, device=dev) * 2 - 1
    rot = torch.empty_like(psi)
    skgemm.drot_band_dev(nd, nb, psi, q, rot)
    skgemm.stream_status()
    assert bool(torch.isfinite(rot).all())
    del psi, q, rot

    nd, nb = 110592, 512

    # Layout kernels (HBM-bound).
    dense = torch.randn(nd, nb, generator=g, dtype=torch.float64, device=dev) / nd ** 0.5
    band16 = torch.empty(nd * nb, dtype=torch.float64, device=dev)
    band32 = torch.empty_like(band16)
    grid = torch.empty_like(band16)
    back = torch.empty_like(band16)
    skgemm.pack_dev(nb, nd, dense, 1, nb, 16, band16)
    skgemm.pack_dev(nb, nd, dense, 1, nb, 32, band32)
    skgemm.band_to_grid_dev(nd, nb, band16, grid)
    skgemm.grid_to_band_dev(nd, nb, grid, back)
    skgemm.stream_status()
    assert torch.equal(back, band16)
    colmajor = torch.empty_like(band16)
    skgemm.unpack_c16_dev(nd, nb, grid, colmajor)
    skgemm.stream_status()
    assert torch.equal(colmajor.view(nb, nd).t(), dense)

    # The rotation on band-packed Psi (no grid-packed copy), native and Ozaki.
    q = torch.rand(nb * nb, generator=g, dtype=torch.float64, device=dev) * 2 - 1
    rot_g = torch.empty_like(band16)
    rot_b = torch.empty_like(band16)
    for prec in (None, skgemm.PREC_OZAKI_I8):
        skgemm.drot_dev(nd, nb, grid, q, rot_g, precision=prec)
        skgemm.drot_band_dev(nd, nb, band16, q, rot_b, precision=prec)
        skgemm.stream_status()
        assert torch.equal(rot_b, rot_g)

    # H Psi producer: periodic halo of band-packed Psi (48^3 grid points, the
    # nd above), then the 6th-order stencil into the GEMM's 32-band-packed B.
    n = 48
    assert n ** 3 == nd
    cx = [0.0, -1.0 / 12, 2.0 / 3, -2.5, 8.0 / 3, -1.0 / 4, 1.0 / 30]
    ext = torch.empty((nb + 15) // 16 * (n + 12) ** 3 * 16, dtype=torch.float64, device=dev)
    a_diag = torch.rand(nd, generator=g, dtype=torch.float64, device=dev)
    hpsi = torch.empty_like(band16)
    skgemm.halo_periodic_dev(n, n, n, nb, band16, ext)
    skgemm.stencil_ext_dev(n, n, n, nb, ext, a_diag, cx, cx, cx, -0.5, hpsi, 32)
    skgemm.stream_status()
    assert bool(torch.isfinite(hpsi).all())

    # Nonlocal projector: H Psi += V_nloc Psi (64 atoms x 2 images).
    rng = np.random.default_rng(8)
    atoms, images, nrow, ncol = 64, 2, 800, 16
    nproj = atoms * images
    proj = skgemm.NlocProjector(
        np.full(nproj, nrow), np.full(nproj, ncol), np.repeat(np.arange(1, atoms + 1), images),
        np.append(np.repeat(np.arange(atoms) * ncol, images), atoms * ncol),
        np.concatenate([rng.permutation(nd)[:nrow] for _ in range(nproj)]),
        rng.uniform(-1, 1, nproj * nrow * ncol), rng.uniform(-0.5, 0.5, nproj * ncol), nd)
    proj.apply(nb, 0.01, band16, hpsi, 32)
    skgemm.stream_status()
    assert bool(torch.isfinite(hpsi).all())
    proj.close()
    del ext, hpsi

    # K = 0 epilogues.
    n = 4096
    d = torch.empty(n * n, dtype=torch.float64, device=dev)
    a0 = torch.zeros(16, dtype=torch.float64, device=dev)
    skgemm.dgemm_packed_dev(n, n, 0, a0, a0, d, n, 1.0, 2.5)
    skgemm.stream_status()
    assert bool((d == 2.5).all())
    skgemm.dgemm_packed_dev_noalloc(n, n, 0, a0, a0, d, n, 1.0, -1.5)
    assert bool((d == -1.5).all())

    # Host-pointer GEMM with a long reduction: k-chunked upload, partial
    # outputs combined by sum_parts_kernel.
    m2, k2 = 2048, 32768
    ah = np.random.default_rng(3).uniform(-1, 1, (m2 // 16) * 16 * k2)
    bh = np.random.default_rng(4).uniform(-1, 1, (m2 // 32) * 32 * k2)
    dh = np.zeros(m2 * m2)
    skgemm.gemm.compute_packed(m2, m2, k2, ah, bh, dh, 1.0, 0.5)
    assert np.isfinite(dh).all()

    # Exact int8 GEMM (lane-scheduled tcgen05 kernel + slab sum).
    ai = torch.randint(-128, 128, (n, n), generator=g, dtype=torch.int8, device=dev)
    bi = torch.randint(-128, 128, (n, n), generator=g, dtype=torch.int8, device=dev)
    ci = torch.empty(n, n, dtype=torch.int32, device=dev)
    skgemm.igemm_s8_dev(n, n, n, ai, n, bi, n, ci, n)
    skgemm.stream_status()
    rows = torch.randint(0, n, (64,), generator=g, device=dev)
    ref = ai[rows].to(torch.float64) @ bi.to(torch.float64).T
    assert torch.equal(ci[rows].to(torch.float64), ref)

    # BF16 Ozaki kernels (results equal the INT8 variant's).
    h = torch.empty(nd * nb, dtype=torch.float64, device=dev)
    skgemm.pack_dev(nb, nd, torch.randn(nd, nb, generator=g, dtype=torch.float64, device=dev)
                    / nd ** 0.5, 1, nb, 32, h)
    hs_b = torch.empty(nb * nb, dtype=torch.float64, device=dev)
    hs_i = torch.empty_like(hs_b)
    skgemm.dgemm_packed_dev(nb, nb, nd, band16, h, hs_b, nb, precision=skgemm.PREC_OZAKI_BF16)
    skgemm.dgemm_packed_dev(nb, nb, nd, band16, h, hs_i, nb, precision=skgemm.PREC_OZAKI_I8)
    q = torch.rand(nb * nb, generator=g, dtype=torch.float64, device=dev) * 2 - 1
    skgemm.drot_dev(nd, nb, grid, q, back, precision=skgemm.PREC_OZAKI_BF16)
    skgemm.stream_status()
    assert torch.equal(hs_b, hs_i)

    # Serving input generators.
    trace = [(0.0, 65536, 256, 1), (0.0, 20000, 128, 2)]
    rows_, _ = skgemm.serve(trace, precision=skgemm.PREC_NATIVE, hbm_budget=20e9,
                            realtime=False)
    assert len(rows_) == 2

    # Peak probes.
    fp64 = skgemm.probe_fp64_peak()
    i8 = skgemm.probe_i8_peak()
    print(f"kernel tour ok: FP64 DMMA peak {fp64:.1f} TFLOP/s, INT8 peak {i8:.0f} TOP/s")



# ------------------------------------------------------------- CPU arm
def _ref_sample(kslice: int):
    """Inputs for a K-sliced sample of the workload: the first `kslice` grid
    points of Psi / H Psi (SYRK, GEMM) and `kslice` grid rows (rotation)."""
    import numpy as np
    rng = np.random.default_rng(20240611)
    scale = 1.0 / ND ** 0.5
    psi = rng.standard_normal((kslice, NB)) * scale
    hpsi = rng.standard_normal((kslice, NB)) * scale
    q = rng.uniform(-1, 1, (NB, NB))
    import oracle
    band = oracle.pack(np.ascontiguousarray(psi.T), 16).ravel()
    h32 = oracle.pack(np.ascontiguousarray(hpsi.T), 32).ravel()
    grid = oracle.grid_pack(psi).ravel()
    return band, h32, grid, np.ascontiguousarray(q).ravel()


def cpu_step_reference(kslice, inputs):
    """One sample step on the reference's own kernels (oracle/_ref, all cores):
    sme_syrk<double>::compute, gemm<double>::compute_packed, sme_gemm_trp_3d."""
    import ctypes
    import numpy as np
    import oracle
    band, h32, grid, q = inputs
    dp = ctypes.POINTER(ctypes.c_double)
    sy = oracle.ref("sme_syrk").ref_sme_syrk_compute
    sy.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_double]
    gm = oracle.ref("gemm_opt").ref_gemm_opt_compute_packed
    gm.argtypes = [ctypes.c_int] * 3 + [dp] * 3 + [ctypes.c_double] * 2
    rt = oracle.ref("trp_3d").ref_trp_3d_compute
    rt.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    S = np.zeros(NB * NB)
    Hs = np.zeros(NB * NB)
    P = np.zeros(kslice * NB)
    t = time.perf_counter()
    sy(kslice, NB, oracle.ptr(band), oracle.ptr(S), 1.0, 0.0)
    gm(NB, NB, kslice, oracle.ptr(band), oracle.ptr(h32), oracle.ptr(Hs), 1.0, 0.0)
    rt(kslice, NB, oracle.ptr(grid), oracle.ptr(q), oracle.ptr(P))
    return time.perf_counter() - t


def cpu_baseline(sample_seconds=10.0, kslice=ND):
    """The reference's own kernels (oracle/_ref) on the host cores, on the full
    workload (or a K-slice of it), repeated until about `sample_seconds`."""
    import oracle
    if not oracle.have_ref():
        return None
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    inputs = _ref_sample(kslice)
    times = [cpu_step_reference(kslice, inputs)]
    while sum(times) < sample_seconds and len(times) < 20:
        times.append(cpu_step_reference(kslice, inputs))
    flops = (NB * (NB + 1) + 2 * NB * NB) * kslice + 2 * kslice * NB * NB
    return {"value": round(flops * len(times) / sum(times) / 1e12, 6), "unit": "TFLOP/s",
            "cores": cores, "kind": "reference",
            "sample": f"{len(times)} passes of the three ops on {kslice} of {ND} grid points; "
                      f"reference kernels sme_syrk.hpp / gemm_opt.cpp / sme_trp_3d.hpp built "
                      f"-O3 (AVX2) with the host SME-intrinsic emulation, OpenMP {cores} threads",
            "seconds": round(sum(times), 3), "cpu_model": cpu_model(),
            "host_has_sme": host_has_sme(),
            "also": cpu_naive_baselines()}


def host_has_sme() -> bool:
    """Arm SME on this host (aarch64 `Features: ... sme`; the x86 `sme` flag
    is AMD's memory encryption and does not count)."""
    import platform
    if platform.machine() not in ("aarch64", "arm64"):
        return False
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("Features") and "sme" in line.split(":", 1)[1].split():
                return True
    except OSError:
        pass
    return False


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def naive_pass(L, kslice, threads, inputs):
    """One pass of the reference's portable naive loops (gemm_opt.cpp:467-475,
    syrk_crsp.cpp:355-373, trp_3d_test.cpp:55-66, as restated in the oracle)
    on a K-slice of the workload; returns seconds."""
    import oracle
    A_col, B_row, A16, grid, q, D, C, P = inputs
    p = oracle.ptr
    t = time.perf_counter()
    L.oracle_syrk_naive(kslice, NB, p(A16), p(C), 1.0, 0.0, threads)
    L.oracle_gemm_naive(NB, NB, kslice, p(A_col), p(B_row), p(D), 1.0, 0.0, threads)
    L.oracle_rot_naive(kslice, NB, p(grid), p(q), p(P), threads)
    return time.perf_counter() - t


def cpu_naive_baselines(target_s=6.0):
    """The reference's portable naive loops built -O3 -march=native on this
    host: serial on 1 core (as the reference runs them), and the same loops
    with their outer loop split over all cores by OpenMP (a restatement, not
    the reference's code). Each times a K-slice of the workload sized to about
    target_s seconds; TFLOP/s are per flop of that slice (the loops' cost is
    linear in K, so it extrapolates to the full 110592 grid points)."""
    import numpy as np
    import oracle
    try:
        L = oracle.naive_native()
    except Exception as e:  # no compiler on this host
        return [{"unavailable": f"naive loops not built: {e}"}]
    cores = os.cpu_count() or 1
    out = []
    for threads, label in ((1, "reference portable naive loops, serial (1 core)"),
                           (cores, f"OpenMP outer-loop restatement of the naive loops "
                                   f"({cores} cores)")):
        ks = 256
        while True:
            rng = np.random.default_rng(5)
            X = rng.standard_normal((ks, NB)) / ND ** 0.5
            Y = rng.standard_normal((ks, NB)) / ND ** 0.5
            inputs = (np.ascontiguousarray(X).ravel(),    # A col-major: A[i + k M] = X[k, i]
                      np.ascontiguousarray(Y).ravel(),    # B row-major: B[k N + j] = Y[k, j]
                      oracle.pack(np.ascontiguousarray(X.T), 16).ravel(),
                      oracle.grid_pack(X).ravel(), rng.uniform(-1, 1, NB * NB),
                      np.zeros(NB * NB), np.zeros(NB * NB), np.zeros(ks * NB))
            sec = naive_pass(L, ks, threads, inputs)
            if sec >= target_s / 4 or ks >= ND:
                break
            ks = min(ND, int(ks * min(8.0, max(2.0, target_s / max(sec, 1e-3)))) // 16 * 16)
        flops = (NB * (NB + 1) + 2 * NB * NB) * ks + 2 * ks * NB * NB
        out.append({"value": round(flops / sec / 1e12, 6), "unit": "TFLOP/s", "cores": threads,
                    "kind": "port", "label": label,
                    "sample": f"the three ops on a {ks}-grid-point slice of {ND} "
                              f"(per-flop rate; the loops are linear in K), -O3 -march=native",
                    "seconds": round(sec, 3)})
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    # Each step is the full workload unless steps * (one step) would exceed
    # about 150 s; then each step is the same K-slice of it.
    ks = ND
    inputs = _ref_sample(ks)
    t1 = cpu_step_reference(ks, inputs)
    if (args.steps + args.warmup) * t1 > 150.0:
        ks = max(1024, int(ND * 150.0 / ((args.steps + args.warmup) * t1)) // 16 * 16)
        inputs = _ref_sample(ks)
    for _ in range(max(0, args.warmup - 1)):
        cpu_step_reference(ks, inputs)
    times = [cpu_step_reference(ks, inputs) for _ in range(args.steps)]
    flops = (NB * (NB + 1) + 2 * NB * NB) * ks + 2 * ks * NB * NB
    tot = sum(times)
    v = flops * len(times) / tot / 1e12
    sample = (f"each step: the three ops on {ks} of {ND} grid points, reference kernels "
              f"(oracle/_ref) with {cores} OpenMP threads")
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 6), "unit": "TFLOP/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(tot / len(times) * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "Nd": ND, "nb": NB,
                       "ops": ["syrk", "gemm", "rotation"], "sample_grid_points": ks,
                       "device": f"host CPU, {cores} cores (the arm launched for {args.gpus} "
                                 f"GPU(s); rank 0 alone runs)"},
            "cpu_baseline": {"value": round(v, 6), "unit": "TFLOP/s", "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(v, 6), "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ batched arm
def batched_instances(n, seed=2024):
    """(grid points, states) of the k-point batch: grid from {24^3, 32^3, 40^3,
    48^3, 64^3}, states log-uniform in [64, 1024]."""
    import numpy as np
    rng = np.random.default_rng(seed)
    grids = [24 ** 3, 32 ** 3, 40 ** 3, 48 ** 3, 64 ** 3]
    out = []
    for _ in range(n):
        ng = int(rng.choice(grids))
        nb = int(round(float(np.exp(rng.uniform(np.log(64), np.log(1024))))))
        out.append((ng, nb))
    return out


def run_batched(args):
    import numpy as np
    import torch
    import skgemm
    rank, world, dist = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    shapes = batched_instances(args.instances)
    if args.max_grid:
        shapes = [(min(ng, args.max_grid), nb) for ng, nb in shapes]
    g = torch.Generator(device=dev).manual_seed(7 + rank)
    items, keep, flop = [], [], 0.0
    for ng, nb in shapes:
        # Packed buffers filled directly: their entries are the matrix entries
        # (N(0,1)/sqrt(Ng)); padding columns only feed outputs that are not stored.
        p16 = torch.randn(((nb + 15) // 16) * 16 * ng, generator=g, dtype=torch.float64,
                          device=dev) / ng ** 0.5
        h32 = torch.randn(((nb + 31) // 32) * 32 * ng, generator=g, dtype=torch.float64,
                          device=dev) / ng ** 0.5
        S = torch.zeros(nb * nb, dtype=torch.float64, device=dev)
        Hs = torch.zeros_like(S)
        keep.append((p16, h32, S, Hs))
        items += [skgemm.batch_item(skgemm.OP_SYRK_PACKED, nb, nb, ng, p16, 0, S, nb),
                  skgemm.batch_item(skgemm.OP_GEMM_PACKED, nb, nb, ng, p16, h32, Hs, nb)]
        flop += nb * nb * ng + 2.0 * nb * nb * ng
    stream = torch.cuda.current_stream()
    if args.precision == "both":
        args.precision = "native"
    prec = {"native": skgemm.PREC_NATIVE, "ozaki": skgemm.PREC_OZAKI_I8,
            "ozaki_bf16": skgemm.PREC_OZAKI_BF16,
            "auto": skgemm.PREC_AUTO}[args.precision]
    plan = skgemm.Plan(items, tile=args.tile, order=2 if args.no_tune else 0,
                       tune=not args.no_tune, stream=stream, precision=prec)
    cfg = plan.config
    peak = skgemm.probe_fp64_peak()
    for _ in range(args.warmup):
        plan.run(stream)
    plan.status(stream)
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(dist)
    clocks.start()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for i in range(args.steps):
        plan.run(stream)
        evs[i + 1].record(stream)
    barrier(dist)
    clk = clocks.stop()
    plan.status(stream)
    per = np.array([evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)])
    total_ms = max_over_ranks(float(per.sum()), dist)
    achieved = flop / (per.mean() * 1e-3) / 1e12
    mem = sum(x.numel() * 8 for k in keep for x in k)
    line = {
        "metric": METRIC, "value": round(job_throughput(flop, args.steps, world, total_ms), 3),
        "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"kpoint_batch_{args.instances}x_syrk_gemm"
                               + (f"_grid_le_{args.max_grid}" if args.max_grid else ""),
                   "instances": args.instances, "flop_per_step": flop,
                   "bytes_resident": mem, "tile": cfg["tile"], "grid": cfg["grid"],
                   "order": cfg["order"], "candidates_timed": cfg["candidates_timed"],
                   "model_efficiency": round(cfg["model_efficiency"], 4),
                   "precision": args.precision, "ozaki_problems": cfg["ozaki_problems"],
                   "launch": "one CUDA graph per step: the grouped persistent Stream-K "
                             "launch (+ the Ozaki kernels of the problems sent there)",
                   "l2": "inputs larger than L2", "parallelism": f"replicas{world}"},
        "latency_ms": {"p50": round(float(np.percentile(per, 50)), 3),
                       "p99": round(float(np.percentile(per, 99)), 3)},
        "roofline": {"bound": "tensor", "achieved": round(achieved, 3), "peak": round(peak, 3),
                     "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                     "peak_source": "measured FP64 DMMA peak (skgemm_probe_fp64_peak, this run)",
                     "kernel": "fp64_grouped_kernel" if cfg["ozaki_problems"] == 0 else
                     "fp64_grouped_kernel + Ozaki split, FP64-equivalent flops",
                     "traffic": None},
        "clocks": clk, "gpu_launches": cfg["graph_kernels"] * args.steps,
    }
    plan.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ------------------------------------------------------------ serving arm
def serve_measure(args, name, requests, rank, dist, policy_name=None):
    """One Poisson trace (200 requests/s, seeded per rank) through the serving
    engine at precision `name`, after a small warm-up trace. Returns the
    engine's throughput, p50/p99 latency (overall and per decile of request
    work), the clocks and the engine's figures."""
    import numpy as np
    import torch
    import skgemm
    prec = {"native": skgemm.PREC_NATIVE, "ozaki": skgemm.PREC_OZAKI_I8}[name]
    trace = skgemm.serve_trace(requests, rate=200.0, seed=11 + rank)
    warm = skgemm.serve_trace(8, rate=200.0, seed=99, nb_range=(32, 256), ng_range=(1e4, 5e4))
    skgemm.serve(warm, precision=prec, hbm_budget=150e9)
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(dist)
    clocks.start()
    policy = {"smallest": skgemm.SERVE_SMALLEST, "fifo": skgemm.SERVE_FIFO,
              "ratio": skgemm.SERVE_RATIO}[policy_name or args.serve_policy]
    rows, o = skgemm.serve(trace, precision=prec, hbm_budget=150e9, realtime=True,
                           policy=policy, aging_s=args.serve_aging,
                           ozaki_streams=args.ozaki_streams)
    barrier(dist)
    clk = clocks.stop()
    lat = np.array([d - a for a, _, d in rows]) * 1e3
    work = np.array([5.0 * nb * nb * ng for _, ng, nb, _ in trace])
    dec = np.minimum(9, (np.argsort(np.argsort(work)) * 10) // len(work))
    p99_dec = [round(float(np.percentile(lat[dec == d], 99)), 1) for d in range(10)
               if np.any(dec == d)]
    return {"precision": name, "requests": requests, "flop": o.flop,
            "makespan_s": round(o.makespan_s, 3),
            "tflops": round(o.flop / o.makespan_s / 1e12, 3),
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 2),
                           "p99": round(float(np.percentile(lat, 99)), 2),
                           "mean": round(float(lat.mean()), 2),
                           "p99_by_work_decile": p99_dec},
            "admission": {"smallest": "least work first, aged (wait / %g s)" % args.serve_aging,
                          "fifo": "arrival order",
                          "ratio": "highest response ratio next (wait / work)"}[
                              policy_name or args.serve_policy],
            "ozaki_streams": args.ozaki_streams if name == "ozaki" else None,
            "batches": o.batches, "mean_batch_problems": round(o.mean_batch_problems, 2),
            "peak_admitted_bytes": o.peak_admitted_bytes, "scratch_bytes": o.scratch_bytes,
            "clocks": clk}


def run_serving(args):
    import skgemm
    if args.precision in ("auto", "ozaki_bf16"):
        raise SystemExit("the serving workload runs --precision native or ozaki")
    name = "native" if args.precision == "both" else args.precision
    rank, world, dist = dist_setup(args.gpus)
    r = serve_measure(args, name, args.requests, rank, dist)
    span = max_over_ranks(r["makespan_s"], dist)
    peak = skgemm.probe_fp64_peak()
    tf = r["tflops"]
    line = {
        "metric": METRIC, "value": round(r["flop"] * world / span / 1e12, 3), "unit": "TFLOP/s",
        "n_gpus": world, "steps": args.requests, "warmup": 8,
        "ms_per_step": round(span / max(1, args.requests) * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"serving_poisson200_{args.requests}req",
                   "precision": name, "arrival_rate_per_s": 200.0,
                   "ozaki_streams": r["ozaki_streams"], "admission": r["admission"],
                   "grid_points": "log-uniform [1e4, 4e5], multiple of 16",
                   "states": "log-uniform [32, 2048], multiple of 16",
                   "hbm_budget_bytes": 150e9, "flop": r["flop"],
                   "batches": r["batches"], "mean_batch_problems": r["mean_batch_problems"],
                   "peak_admitted_bytes": r["peak_admitted_bytes"],
                   "scratch_bytes": r["scratch_bytes"], "parallelism": f"replicas{world}"},
        "latency_ms": r["latency_ms"],
        "roofline": {"bound": "tensor", "achieved": round(tf, 3), "peak": round(peak, 3),
                     "unit": "TFLOP/s", "frac": round(tf / peak, 4),
                     "peak_source": "measured FP64 DMMA peak (skgemm_probe_fp64_peak, this run)",
                     "kernel": "fp64_grouped_kernel" if name == "native" else "i8_gemm_kernel",
                     "traffic": None},
        "clocks": r["clocks"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.workload == "tour":
        run_tour(args)
    elif args.workload == "op":
        run_op(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
