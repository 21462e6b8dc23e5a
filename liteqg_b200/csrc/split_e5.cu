// Split search kernel instances with a 160-slot sorted array (E = 5).
#include "split_kernel.cuh"

namespace lqg {
template cudaError_t split_dispatch<5>(const SearchArgs&, const ReplayArgs&, int, int, int, int,
                                        cudaStream_t, int*);
}  // namespace lqg
