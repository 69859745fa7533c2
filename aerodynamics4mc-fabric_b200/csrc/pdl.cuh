// Programmatic dependent launch between the kernels of a step (sm_90+): a
// kernel launched with launch_pdl may be scheduled while its predecessor on
// the stream still runs. It must call pdl_wait() before it reads anything the
// predecessor writes; the wait returns once the predecessor grid has
// completed and its memory operations are visible. pdl_trigger() at the top
// of a kernel lets its own dependent be scheduled once every block of this
// grid has started (the dependent's blocks then hold their slots and wait).
// Without the launch attribute, or after a predecessor that never triggers,
// both are no-ops for the ordering: the dependent starts at completion.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace aero {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace aero
