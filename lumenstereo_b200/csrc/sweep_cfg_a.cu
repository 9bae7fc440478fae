// sweep_cfg_a.cu -- compiled instances of the sweep kernel (sweep_kernel.cuh) for
// padded disparity counts 64, 128; one translation unit per group keeps
// the build parallel.
#include "sweep_kernel.cuh"

namespace lumen {

cudaError_t sweep_dispatch_64(SweepArgs a, int T, int NW, bool wrap, bool diag,
                              cudaStream_t s, int numSMs, int* g) {
    if (T == 32 && NW == 4) {
        return diag ? sweep_launch_np<32, 1, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 1, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 32 && NW == 8) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<32, 1, 8, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 1, 8, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 16 && NW == 4) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<16, 2, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<16, 2, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 8 && NW == 4) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<8, 4, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<8, 4, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 8 && NW == 2) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<8, 4, 2, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<8, 4, 2, 1>(a, wrap, s, numSMs, g);
    }
    return cudaErrorInvalidValue;
}

cudaError_t sweep_dispatch_128(SweepArgs a, int T, int NW, bool wrap, bool diag,
                              cudaStream_t s, int numSMs, int* g) {
    if (T == 32 && NW == 4) {
        return diag ? sweep_launch_np<32, 2, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 2, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 32 && NW == 8) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<32, 2, 8, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 2, 8, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 16 && NW == 4) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<16, 4, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<16, 4, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 8 && NW == 4) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<8, 8, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<8, 8, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 8 && NW == 2) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<8, 8, 2, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<8, 8, 2, 1>(a, wrap, s, numSMs, g);
    }
    return cudaErrorInvalidValue;
}

}  // namespace lumen
