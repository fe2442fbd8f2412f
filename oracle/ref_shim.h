// Force-included into every translation unit of the reference build
// (oracle/ref_build.py).  The reference's scan kernel (main.cu:35-39) reads
// visited[v] before testing v < V, for v up to the next multiple of its
// 262,144-thread grid; every device allocation is therefore padded by 4 MiB
// so those reads stay inside the allocation.  Nothing else changes.
#pragma once
#include <cuda_runtime.h>

template <class T>
static inline cudaError_t dc_ref_padded_malloc(T** p, size_t bytes) {
    return cudaMalloc(reinterpret_cast<void**>(p), bytes + (size_t(4) << 20));
}
#define cudaMalloc dc_ref_padded_malloc
