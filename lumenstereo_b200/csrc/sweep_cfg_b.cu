// sweep_cfg_b.cu -- compiled instances of the sweep kernel (sweep_kernel.cuh) for
// padded disparity counts 192, 256; one translation unit per group keeps
// the build parallel.
#include "sweep_kernel.cuh"

namespace lumen {

cudaError_t sweep_dispatch_192(SweepArgs a, int T, int NW, bool wrap, bool diag,
                              cudaStream_t s, int numSMs, int* g) {
    if (T == 32 && NW == 4) {
        return diag ? sweep_launch_np<32, 3, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 3, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 32 && NW == 8) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<32, 3, 8, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 3, 8, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 16 && NW == 4) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<16, 6, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<16, 6, 4, 1>(a, wrap, s, numSMs, g);
    }
    return cudaErrorInvalidValue;
}

cudaError_t sweep_dispatch_256(SweepArgs a, int T, int NW, bool wrap, bool diag,
                              cudaStream_t s, int numSMs, int* g) {
    if (T == 32 && NW == 4) {
        return diag ? sweep_launch_np<32, 4, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 4, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 32 && NW == 8) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<32, 4, 8, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 4, 8, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 16 && NW == 4) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<16, 8, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<16, 8, 4, 1>(a, wrap, s, numSMs, g);
    }
    return cudaErrorInvalidValue;
}

}  // namespace lumen
