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

// Allow a kernel every dynamic shared memory size the device offers beside
// its static shared memory.  The attribute belongs to the function, not to
// a launch: host threads that launch one kernel with different sizes
// (handles on one device) would undo each other's per-size setting, so it
// is always set to the same maximum.
template <class K>
inline cudaError_t allow_smem(K kernel) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    int optin = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - int(fa.sharedSizeBytes));
    if (e != cudaSuccess) cudaGetLastError();     // reported by the return value, not left behind
    return e;
}

}  // namespace elas
