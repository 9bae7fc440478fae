// pair_t16.cu -- schedule 6 instances with 16-lane rows (padded disparities 192 to 320), 16-row bands.
#include "pair_kernel.cuh"

namespace lumen {
template cudaError_t pair_launch_t<6, 16, 16>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<8, 16, 16>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<10, 16, 16>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<6, 16, 16, false>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<8, 16, 16, false>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
template cudaError_t pair_launch_t<10, 16, 16, false>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
}  // namespace lumen
