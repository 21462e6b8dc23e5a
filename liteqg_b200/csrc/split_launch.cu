// Dispatch of the split search kernel over its sorted-array instances.
#include "split_kernel.cuh"

namespace lqg {

#define LQG_SPLIT_EXTERN(E)                                                                   \
    extern template cudaError_t split_dispatch<E>(const SearchArgs&, const ReplayArgs&, int, \
                                                  int, int, int, cudaStream_t, int*);
LQG_SPLIT_EXTERN(2)
LQG_SPLIT_EXTERN(3)
LQG_SPLIT_EXTERN(5)
LQG_SPLIT_EXTERN(9)
LQG_SPLIT_EXTERN(17)
#undef LQG_SPLIT_EXTERN

bool split_replays_in_place_host(uint32_t vbits, uint32_t scap, uint32_t rcap) {
    return split_replays_in_place(vbits, scap, rcap);
}

size_t split_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t scap, int warps) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 8 * dpad + (size_t)warps * split_warp_bytes(dim, vbits, scap);
}

cudaError_t launch_split(const SearchArgs& a, const ReplayArgs& ra, int E, int G, int degw,
                         int warps, int blocks, cudaStream_t st, int* occ) {
    switch (E) {
        case 2: return split_dispatch<2>(a, ra, G, degw, warps, blocks, st, occ);
        case 3: return split_dispatch<3>(a, ra, G, degw, warps, blocks, st, occ);
        case 5: return split_dispatch<5>(a, ra, G, degw, warps, blocks, st, occ);
        case 9: return split_dispatch<9>(a, ra, G, degw, warps, blocks, st, occ);
        case 17: return split_dispatch<17>(a, ra, G, degw, warps, blocks, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lqg
