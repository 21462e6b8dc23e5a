// Split search kernel instances with a 64-slot sorted array (E = 2).
#include "split_kernel.cuh"

namespace lqg {
template cudaError_t split_dispatch<2>(const SearchArgs&, const ReplayArgs&, int, int, int, int,
                                        cudaStream_t, int*);
}  // namespace lqg
