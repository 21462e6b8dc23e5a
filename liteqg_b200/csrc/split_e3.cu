// Split search kernel instances with a 96-slot sorted array (E = 3).
#include "split_kernel.cuh"

namespace lqg {
template cudaError_t split_dispatch<3>(const SearchArgs&, const ReplayArgs&, int, int, int, int,
                                        cudaStream_t, int*);
}  // namespace lqg
