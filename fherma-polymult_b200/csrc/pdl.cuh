// Programmatic dependent launch: a kernel launched this way may start while the
// kernel before it on the stream is still finishing its last wave.  It runs
// whatever does not touch the predecessor's outputs (barrier set-up, TMEM
// allocation, loads of read-only plan tables), then waits for the predecessor
// to complete before its first access to shared buffers.  Each kernel also
// lets its own successor launch as soon as all of its blocks are running.
// Both device calls are no-ops in a grid launched without the attribute.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace fpm {

__device__ __forceinline__ void pdl_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Blocks until the preceding grid has completed and its writes are visible.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace fpm
