// Replay search kernel instances with a 544-slot sorted pool (E = 17).
#include "replay_kernel.cuh"

namespace lqg {
template cudaError_t replay_dispatch<17>(const SearchArgs&, const ReplayArgs&, int, int, int,
                                         cudaStream_t, int*);
}  // namespace lqg
