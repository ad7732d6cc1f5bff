// fcb_launch.cuh -- programmatic dependent launch of the advance's kernels.
//
// An advance is a chain of dependent launches on one stream (level updates,
// ghost-fill stages, time sync, time interpolation), most of them a few
// microseconds long, so the gap between the end of one grid and the start of
// the next is a large part of a step.  With programmatic stream serialization
// the next grid is scheduled once every CTA of the running grid has executed
// griddepcontrol.launch_dependents (or exited); its CTAs then sit at
// griddepcontrol.wait, which returns when the previous grid has completed and
// its memory operations are visible.  Every kernel launched this way calls
// grid_dependency_wait() before its first global memory access, so the stream
// order of all reads and writes is that of plain launches; only the launch gap
// is hidden.  In a kernel launched without the attribute both instructions
// are no-ops.
#pragma once
#include <cuda_runtime.h>
#include <utility>

namespace fcb {

__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Host flag of the calling thread: launches through launch_k carry the
// programmatic-serialization attribute while it is set (ProgrammaticScope).
bool programmatic_launch();

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                            Args&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = programmatic_launch() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

}  // namespace fcb
