// Programmatic dependent launch for the chain of passes of a field evaluation.  A kernel
// launched with launch_pdl may become resident while its predecessor's last blocks run;
// it must begin with pdl_begin(): the trigger lets the next kernel of the chain launch
// early in turn, and the wait returns once the predecessor has completed and its writes
// are visible, so nothing the predecessor writes is read before it.  MM_PDL=0 in the
// environment launches every kernel the ordinary way; a plan can also turn it off for its
// own launches (PdlScope).
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>

namespace mm {

__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

inline bool pdl_env() {
    static const bool on = [] {
        const char* e = getenv("MM_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

// The calling thread's current choice: -1 outside any scope (the environment decides),
// else 0 / 1 as set by the innermost PdlScope.
inline thread_local int g_pdl_scope = -1;

inline bool pdl_enabled() { return pdl_env() && g_pdl_scope != 0; }

// Sets the choice for the launches made while it lives (on this host thread).
struct PdlScope {
    int saved;
    explicit PdlScope(bool on) : saved(g_pdl_scope) { g_pdl_scope = on ? 1 : 0; }
    ~PdlScope() { g_pdl_scope = saved; }
    PdlScope(const PdlScope&) = delete;
    PdlScope& operator=(const PdlScope&) = delete;
};

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
