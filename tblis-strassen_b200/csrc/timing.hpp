// Optional per-kernel CUDA-event timing (off by default).  When enabled with
// tblis_stra_set_kernel_timing(1), every kernel launch of the library is
// bracketed by two events on its own stream; tblis_stra_kernel_timing() sums
// the elapsed times per kernel kind.  Used by the benchmark to report the
// dominant kernel's time inside a full run.
#pragma once

#include <cuda_runtime.h>

namespace tsb {

enum KernelKind
{
    KK_FUSED = 0,        // stra_dmma_kernel (fused gathers and sums)
    KK_PACK = 1,         // pack_kernel
    KK_PACKED_GEMM = 2,  // packed_gemm_kernel
    KK_AUX = 3,          // scale / sum-gather / scatter-add
    KK_SPLIT_GEMM = 4,   // split_gemm_kernel (tcgen05, FP32 via bf16 planes)
    KK_FUSED_TMA = 5,    // stra_fused_pair_kernel, tensor-map producer
    KK_FUSED_PAIRS = 6,  // stra_fused_pair_kernel, 16-byte pair-copy producer
    KK_COUNT = 7
};

bool timing_enabled();
void timing_begin(int kind, cudaStream_t stream);
void timing_end(int kind, cudaStream_t stream);

}  // namespace tsb
