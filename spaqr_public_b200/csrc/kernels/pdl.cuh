// Programmatic dependent launch of the factorization and sweep kernels: every
// kernel launched with launch_pdl (or with the same attribute) starts with
// pdl_enter(), which waits until the grids it depends on have completed and
// their writes are visible (griddepcontrol.wait, a no-op without the launch
// attribute), then lets the next kernel of the stream begin launching once all
// of this grid's CTAs have started (griddepcontrol.launch_dependents). The
// next kernel's CTAs then take the SMs this grid's last CTAs leave free,
// instead of starting only after this grid has drained.
#pragma once

#include <cuda_runtime.h>

namespace spq {

__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// kernel<<<grid, block, smem, s>>>(args...) with the programmatic stream
// serialization attribute and, for cluster > 0, the cluster dimension.
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       unsigned cluster, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    int na = 0;
    at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
    if (cluster > 0) {
        at[na].id = cudaLaunchAttributeClusterDimension;
        at[na].val.clusterDim.x = cluster;
        at[na].val.clusterDim.y = 1;
        at[na].val.clusterDim.z = 1;
        ++na;
    }
    cfg.attrs = at;
    cfg.numAttrs = na;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace spq
