"""The kernel tour (`bench.py --workload tour`: one launch of every auxiliary
kernel, each result checked) runs through on the GPU: layout round trip,
K = 0 fills, the exact int8 GEMM against an FP64 product, BF16 = INT8 Ozaki
results, a two-request serving trace and the peak probes."""
import pytest

pytestmark = pytest.mark.gpu


def test_kernel_tour(cuda):
    import bench
    bench.run_tour()
