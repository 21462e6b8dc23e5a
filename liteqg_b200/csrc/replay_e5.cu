// Replay search kernel instances with a 160-slot sorted pool (E = 5).
#include "replay_kernel.cuh"

namespace lqg {
template cudaError_t replay_dispatch<5>(const SearchArgs&, const ReplayArgs&, int, int, int,
                                         cudaStream_t, int*);
}  // namespace lqg
