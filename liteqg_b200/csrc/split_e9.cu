// Split search kernel instances with a 288-slot sorted array (E = 9).
#include "split_kernel.cuh"

namespace lqg {
template cudaError_t split_dispatch<9>(const SearchArgs&, const ReplayArgs&, int, int, int, int,
                                        cudaStream_t, int*);
}  // namespace lqg
