// Fast search kernel instances with a 512-entry pool (E = 16).
#include "fast_kernel.cuh"

namespace lqg {
template cudaError_t fast_dispatch<16>(const SearchArgs&, int, int, int, int, size_t,
                                       cudaStream_t, int*);
}  // namespace lqg
