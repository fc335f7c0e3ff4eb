// Programmatic dependent launch (sm_90 and later) for chains of small kernels
// captured into CUDA graphs.
//
// A kernel launched with launch_pdl into a capturing stream may be scheduled
// while the kernel before it is still running, so inside the graph the launch
// latency of a chain of short kernels overlaps their execution.  Every kernel
// launched this way calls pdl_begin() first: griddepcontrol.wait returns once
// the preceding grid has completed and its memory writes are visible, and
// griddepcontrol.launch_dependents then lets the next kernel of the chain be
// scheduled.  Both instructions do nothing in a kernel launched without the
// attribute.  Outside a capture launch_pdl makes a plain launch: eager chains
// of feature kernels measured several times slower with the attribute.
#pragma once

#include <utility>

#include <cuda_runtime.h>

namespace csg {

__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... Params, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                              Args&&... args) {
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    const cudaError_t query = cudaStreamIsCapturing(stream, &capture);
    if (query != cudaSuccess) return query;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t config{};
    config.gridDim = grid;
    config.blockDim = block;
    config.dynamicSmemBytes = smem;
    config.stream = stream;
    config.attrs = attr;
    config.numAttrs = capture == cudaStreamCaptureStatusActive ? 1 : 0;
    return cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...);
}

}  // namespace csg
