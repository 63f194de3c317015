// Where an operand's memory lives, as the entry points need to know it.
#pragma once

#include <cuda_runtime.h>

namespace tsb {

// HOST: pageable or pinned host memory (staged through device memory by the
// regular entry points); LOCAL: device memory of `device` or managed memory
// (used in place); OTHER_DEVICE: device memory of another GPU, which a kernel
// on `device` must not dereference (no peer mapping is assumed), so every
// entry point rejects it with TBLIS_STRA_ERR_ARG.
enum class MemKind { HOST, LOCAL, OTHER_DEVICE };

inline MemKind mem_kind(const void* p, int device)
{
    if (!p) return MemKind::HOST;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) { cudaGetLastError(); return MemKind::HOST; }
    if (attr.type == cudaMemoryTypeManaged) return MemKind::LOCAL;
    if (attr.type == cudaMemoryTypeDevice) return attr.device == device ? MemKind::LOCAL : MemKind::OTHER_DEVICE;
    return MemKind::HOST;
}

}  // namespace tsb
