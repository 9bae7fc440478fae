// sweep_cfg_d.cu -- compiled instances of the sweep kernel (sweep_kernel.cuh) for
// padded disparity counts 448, 512; one translation unit per group keeps
// the build parallel.
#include "sweep_kernel.cuh"

namespace lumen {

cudaError_t sweep_dispatch_448(SweepArgs a, int T, int NW, bool wrap, bool diag,
                              cudaStream_t s, int numSMs, int* g) {
    if (T == 32 && NW == 4) {
        return diag ? sweep_launch_np<32, 7, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 7, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 32 && NW == 8) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<32, 7, 8, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 7, 8, 1>(a, wrap, s, numSMs, g);
    }
    return cudaErrorInvalidValue;
}

cudaError_t sweep_dispatch_512(SweepArgs a, int T, int NW, bool wrap, bool diag,
                              cudaStream_t s, int numSMs, int* g) {
    if (T == 32 && NW == 4) {
        return diag ? sweep_launch_np<32, 8, 4, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 8, 4, 1>(a, wrap, s, numSMs, g);
    }
    if (T == 32 && NW == 8) {
        if (wrap) return cudaErrorInvalidValue;
        return diag ? sweep_launch_np<32, 8, 8, 3>(a, wrap, s, numSMs, g)
                    : sweep_launch_np<32, 8, 8, 1>(a, wrap, s, numSMs, g);
    }
    return cudaErrorInvalidValue;
}

}  // namespace lumen
