// Programmatic dependent launch for the chain of passes of a field evaluation.  A kernel
// launched with launch_pdl may become resident while its predecessor's last blocks run;
// it must begin with pdl_begin(): the trigger lets the next kernel of the chain launch
// early in turn, and the wait returns once the predecessor has completed and its writes
// are visible, so nothing the predecessor writes is read before it.  MM_PDL=0 in the
// environment launches every kernel the ordinary way.
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>

namespace mm {

__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

inline bool pdl_enabled() {
    static const bool on = [] {
        const char* e = getenv("MM_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    if (!pdl_enabled()) {
        kern<<<grid, block, smem, st>>>(args...);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

}  // namespace mm
