// Host buffers of the host-pointer entry points (see pm_hostio.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pm {

// Device address of page-locked, mapped host memory, or null for memory the
// GPU cannot read directly (pageable memory, or a failed lookup).
const void* mapped_host(const void* p);

// Copies `bytes` from host memory to device memory `dst` on stream st: a
// streaming kernel when the host buffer is mapped and 16-byte aligned,
// cudaMemcpyAsync otherwise.
cudaError_t copy_in(void* dst, const void* host, size_t bytes, int num_sms, cudaStream_t st);

}  // namespace pm
