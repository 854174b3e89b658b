// Programmatic dependent launch on sm_100a.  A kernel launched with
// launch_pdl may begin (its CTAs become resident and run their set-up) while
// the previous kernel of its stream is still finishing; it executes
// griddep_wait() before its first access to memory that earlier work of the
// stream writes or reads, and that wait returns once the previous kernel has
// completed with its writes visible.  griddep_launch() in a kernel lets the
// next kernel of the stream, if launched with launch_pdl, begin launching
// once every CTA has executed it or exited (no effect on a normal launch).
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace qsk {

__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... P, typename... A>
cudaError_t launch_pdl(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A &&...args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

}  // namespace qsk
