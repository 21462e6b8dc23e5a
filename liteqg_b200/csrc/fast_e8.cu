// Fast search kernel instances with a 256-entry pool (E = 8).
#include "fast_kernel.cuh"

namespace lqg {
template cudaError_t fast_dispatch<8>(const SearchArgs&, int, int, int, int, size_t,
                                       cudaStream_t, int*);
}  // namespace lqg
