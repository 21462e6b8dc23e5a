// Replay search kernel instances with a 288-slot sorted pool (E = 9).
#include "replay_kernel.cuh"

namespace lqg {
template cudaError_t replay_dispatch<9>(const SearchArgs&, const ReplayArgs&, int, int, int,
                                         cudaStream_t, int*);
}  // namespace lqg
