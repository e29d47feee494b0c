// scan.cuh -- exclusive prefix sum of uint32 counts on the device (counting sorts).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace csb {

// Scratch bytes scan_exclusive_u32 needs for n elements.
size_t scan_workspace_bytes(size_t n);
// out[i] = sum_{k<i} in[i]; in and out must not overlap.  No allocation, no sync.
cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, void* tmp,
                               cudaStream_t stream);

}  // namespace csb
