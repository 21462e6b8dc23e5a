// Dispatch of the batched-acceptance search kernel over its instances.
#include "batch_kernel.cuh"

namespace lqg {

#define LQG_BATCH_EXTERN(G)                                                                  \
    extern template cudaError_t batch_dispatch<G>(const SearchArgs&, const ReplayArgs&, int, \
                                                  int, int, cudaStream_t, int*);
LQG_BATCH_EXTERN(2)
LQG_BATCH_EXTERN(4)
LQG_BATCH_EXTERN(8)
#undef LQG_BATCH_EXTERN

bool batch_replays_in_place_host(uint32_t vbits, uint32_t scap, uint32_t acap, uint32_t rcap) {
    return batch_replays_in_place(vbits, scap, acap, rcap);
}

size_t batch_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t scap, uint32_t acap, int warps) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 8 * dpad + (size_t)warps * batch_warp_bytes(dim, vbits, scap, acap);
}

cudaError_t launch_batch(const SearchArgs& a, const ReplayArgs& ra, int G, int degw, int warps,
                         int blocks, cudaStream_t st, int* occ) {
    switch (G) {
        case 2: return batch_dispatch<2>(a, ra, degw, warps, blocks, st, occ);
        case 4: return batch_dispatch<4>(a, ra, degw, warps, blocks, st, occ);
        case 8: return batch_dispatch<8>(a, ra, degw, warps, blocks, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lqg
