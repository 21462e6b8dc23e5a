// Fast search kernel instances with a 64-entry pool (E = 2).
#include "fast_kernel.cuh"

namespace lqg {
template cudaError_t fast_dispatch<2>(const SearchArgs&, int, int, int, int, size_t,
                                       cudaStream_t, int*);
}  // namespace lqg
