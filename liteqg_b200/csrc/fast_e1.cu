// Fast search kernel instances with a 32-entry pool (E = 1).
#include "fast_kernel.cuh"

namespace lqg {
template cudaError_t fast_dispatch<1>(const SearchArgs&, int, int, int, int, size_t,
                                       cudaStream_t, int*);
}  // namespace lqg
