// Kernel launches of the pipeline with programmatic dependent launch (PDL).
//
// A kernel launched with launch_k() may be scheduled while the previous
// kernel of its stream is still running.  Every kernel of this library
// calls grid_dep_wait() before anything else; it returns once all preceding
// work of the stream has completed and its writes are visible, so the
// stream order is unchanged and only launch processing and CTA rampup
// overlap the previous kernel.  (Without the launch attribute the wait
// returns at once.)  ELAS_B200_PDL=0 in the environment launches without it.
#pragma once

#include <cstdlib>
#include <utility>
#include <cuda_runtime.h>

namespace elas {

inline bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("ELAS_B200_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                            Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

}  // namespace elas
