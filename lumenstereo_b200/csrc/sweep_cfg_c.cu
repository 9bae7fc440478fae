// sweep_cfg_c.cu -- compiled instances of the sweep kernel (sweep_kernel.cuh) for
// padded disparity counts 320, 384; one translation unit per group keeps
// the build parallel.
#include "sweep_kernel.cuh"

namespace lumen {

cudaError_t sweep_dispatch_320(SweepArgs a, int T, int NW, bool wrap, bool diag,
                              cudaStream_t s, int numSMs, int* g) {
    if (T == 32 && NW == 4) {
        return diag ? sweep_launch_np<32, 5, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 5, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 32 && NW == 8) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<32, 5, 8, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 5, 8, 1>(a, wrap, s, numSMs, g);
    }
    return cudaErrorInvalidValue;
}

cudaError_t sweep_dispatch_384(SweepArgs a, int T, int NW, bool wrap, bool diag,
                              cudaStream_t s, int numSMs, int* g) {
    if (T == 32 && NW == 4) {
        return diag ? sweep_launch_np<32, 6, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 6, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 32 && NW == 8) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<32, 6, 8, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 6, 8, 1>(a, wrap, s, numSMs, g);
    }
    return cudaErrorInvalidValue;
}

}  // namespace lumen
