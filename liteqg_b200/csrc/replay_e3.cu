// Replay search kernel instances with a 96-slot sorted pool (E = 3).
#include "replay_kernel.cuh"

namespace lqg {
template cudaError_t replay_dispatch<3>(const SearchArgs&, const ReplayArgs&, int, int, int,
                                         cudaStream_t, int*);
}  // namespace lqg
