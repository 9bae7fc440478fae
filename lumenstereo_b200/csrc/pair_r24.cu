// pair_r24.cu -- schedule 6 instances with 24-row bands (8-lane rows for
// padded disparities 64 and 128, 16-lane rows for 192 to 320).
#include "pair_kernel.cuh"

namespace lumen {
template cudaError_t pair_launch_t<4, 8, 24>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<8, 8, 24>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<6, 16, 24>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<8, 16, 24>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<10, 16, 24>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
}  // namespace lumen
