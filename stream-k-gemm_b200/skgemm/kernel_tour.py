"""One launch of every auxiliary kernel of the library on a representative
workload, for profiling (ncu) and as a quick end-to-end exercise:

    python -m skgemm.kernel_tour

Kernels and workloads (inputs larger than L2 where the kernel is HBM-bound):
  pack_kernel<16>, pack_kernel<32>   dense 110592 x 512 -> band-packed (453 MB)
  band_grid_kernel (both ways)       110592 x 512 band <-> grid packed (453 MB)
  unpack_kernel<16>                  grid-packed -> column-major (linalg_unpack_c16)
  fp64_streamk_kernel_ak             the rotation on band-packed Psi, 8192 x 1024
                                     (512 tiles of 128 x 128: the 128-row kernel)
  fp64_streamk_kernel64_ak,          the rotation on band-packed Psi, 110592 x 512,
  norm_partials / convert_tma (KM)   native and Ozaki (K-major operand reads)
  halo_periodic_kernel,              H Psi on the 48^3 grid (= 110592 points) x 512:
  stencil_ext_kernel<32>             periodic halo, then the 6th-order stencil
  nloc_forward / nloc_chi_c /        the nonlocal projector on the same Psi: 64 atoms
  nloc_backward<32>                  x 2 periodic images, 800 rows x 16 columns each
  k0_kernel                          GEMM with K = 0 (D = gamma), 4096 x 4096
  sum_parts_kernel                   the host GEMM's k-chunk combine, 2048 x 2048 x 32768
  noalloc_fill_kernel                the allocation-free GEMM with K = 0
  i8_gemm_kernel + sum_partials      the public exact int8 GEMM, 4096 x 4096 x 4096
  BF16 Ozaki kernels                 GEMM 512 x 512 x 110592, rotation 110592 x 512
  gen_normal / gen_uniform           a two-request serving trace (inputs made on
                                     the device from seeds)
  dmma_peak_kernel, i8_peak_kernel   the peak probes
Every result is checked for a device-side error; nothing here is timed."""
from __future__ import annotations

import numpy as np
import torch

import skgemm


def main() -> None:
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


if __name__ == "__main__":
    np.seterr(all="ignore")
    main()
