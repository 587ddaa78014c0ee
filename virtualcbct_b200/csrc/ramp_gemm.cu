// ramp_gemm.cu -- BF16 3-term split tensor-core ramp filter (tcgen05); see below.
#include "internal.h"

namespace vcbct {

size_t ramp_gemm_workspace_bytes(int V, int H, int W) { (void)V; (void)H; (void)W; return 256; }

cudaError_t launch_ramp_gemm_bf16x3(const float*, float*, const float*, const FilterView*,
                                    const float*, float, float, int, int, int, void*, cudaStream_t)
{
    return cudaErrorNotSupported;
}

}  // namespace vcbct
