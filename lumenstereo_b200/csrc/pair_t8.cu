// pair_t8.cu -- schedule 6 instances with 8-lane rows (padded disparities 64 and 128).
#include "pair_kernel.cuh"

namespace lumen {
template cudaError_t pair_launch_t<4, 8, 16>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<8, 8, 16>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<4, 8, 32>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<8, 8, 32>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<4, 8, 16, false>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<8, 8, 16, false>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
}  // namespace lumen
