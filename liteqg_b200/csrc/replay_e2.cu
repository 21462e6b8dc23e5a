// Replay search kernel instances with a 64-slot sorted pool (E = 2).
#include "replay_kernel.cuh"

namespace lqg {
template cudaError_t replay_dispatch<2>(const SearchArgs&, const ReplayArgs&, int, int, int,
                                         cudaStream_t, int*);
}  // namespace lqg
