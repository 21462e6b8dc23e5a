// Fast search kernel instances with a 128-entry pool (E = 4).
#include "fast_kernel.cuh"

namespace lqg {
template cudaError_t fast_dispatch<4>(const SearchArgs&, int, int, int, int, size_t,
                                       cudaStream_t, int*);
}  // namespace lqg
