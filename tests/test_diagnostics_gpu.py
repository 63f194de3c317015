"""Diagnostics of the library on the GPU: the FP64 tensor-pipe ceiling
measurement and the per-kernel CUDA-event timing the benchmark reads."""
import pytest

pytestmark = pytest.mark.gpu


def test_dmma_ceiling_is_plausible(tsb, cuda):
    before = tsb.launch_count()
    tf, ms = tsb.measure_dmma_peak(4000)
    assert tsb.launch_count() == before + 2
    # B200: about 37 TFLOP/s FP64 at 1.965 GHz; anything far outside means
    # the loop was not doing the work
    assert 10.0 < tf < 60.0, tf
    assert ms > 0.0


def test_kernel_timing_sees_the_gemm(tsb, cuda):
    import torch
    A = torch.rand(1024, 1024, dtype=torch.float64, device=cuda)
    B = torch.rand(1024, 1024, dtype=torch.float64, device=cuda)
    C = torch.zeros(1024, 1024, dtype=torch.float64, device=cuda)
    tsb.set_kernel_timing(True)
    try:
        tsb.contract(1, 1.0, A, "ik", B, "kj", 0.0, C, "ij")
        torch.cuda.synchronize()
        n, ms = tsb.kernel_timing("packed_gemm")
        assert n >= 1 and ms > 0.0
    finally:
        tsb.set_kernel_timing(False)
