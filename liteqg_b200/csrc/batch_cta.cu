// Batched-acceptance search kernel, query-per-block instances (4 warps per
// query, 4 lanes per candidate), for small batches.
#include "batch_kernel.cuh"

namespace lqg {

cudaError_t launch_batch_cta(const SearchArgs& a, const ReplayArgs& ra, int degw, int blocks,
                             cudaStream_t st, int* occ) {
    switch (degw) {
        case 1: return batch_cta_run<1>(a, ra, blocks, st, occ);
        case 2: return batch_cta_run<2>(a, ra, blocks, st, occ);
        case 3: return batch_cta_run<3>(a, ra, blocks, st, occ);
        case 4: return batch_cta_run<4>(a, ra, blocks, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lqg
