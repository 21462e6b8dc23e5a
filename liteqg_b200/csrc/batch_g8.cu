// Batched-acceptance search kernel instances with 8 lanes per candidate.
#include "batch_kernel.cuh"

namespace lqg {
template cudaError_t batch_dispatch<8>(const SearchArgs&, const ReplayArgs&, int, int, int,
                                       cudaStream_t, int*);
}  // namespace lqg
