// pair_wide.cu -- schedule 6 instances with wider lane teams for padded
// disparities 64 and 128 (16 or 32 lanes per row, 16-row bands): fewer words
// per lane and more warps per band than the 8-lane default.
#include "pair_kernel.cuh"

namespace lumen {
template cudaError_t pair_launch_t<2, 16, 16>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<4, 16, 16>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<2, 32, 16>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
}  // namespace lumen
