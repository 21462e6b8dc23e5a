// Split search kernel instances with a 544-slot sorted array (E = 17).
#include "split_kernel.cuh"

namespace lqg {
template cudaError_t split_dispatch<17>(const SearchArgs&, const ReplayArgs&, int, int, int, int,
                                        cudaStream_t, int*);
}  // namespace lqg
