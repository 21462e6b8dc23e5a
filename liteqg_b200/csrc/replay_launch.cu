// Dispatch of the replay search kernel over its pool-size instances.
#include "replay_kernel.cuh"

namespace lqg {

extern template cudaError_t replay_dispatch<2>(const SearchArgs&, const ReplayArgs&, int, int,
                                               int, cudaStream_t, int*);
extern template cudaError_t replay_dispatch<3>(const SearchArgs&, const ReplayArgs&, int, int,
                                               int, cudaStream_t, int*);
extern template cudaError_t replay_dispatch<5>(const SearchArgs&, const ReplayArgs&, int, int,
                                               int, cudaStream_t, int*);
extern template cudaError_t replay_dispatch<9>(const SearchArgs&, const ReplayArgs&, int, int,
                                               int, cudaStream_t, int*);
extern template cudaError_t replay_dispatch<17>(const SearchArgs&, const ReplayArgs&, int, int,
                                                int, cudaStream_t, int*);

// Smallest instance whose sorted pool holds ef entries plus 32 ties at the bound.
int replay_pool_regs(uint32_t ef_max) {
    const int es[] = {2, 3, 5, 9, 17};
    for (int e : es)
        if (32u * e - 32u >= ef_max) return e;
    return 0;
}

size_t replay_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t rcap, uint32_t scap, int swarps) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 8 * dpad + (size_t)swarps * replay_warp_bytes(dim, vbits, rcap, scap);
}

cudaError_t launch_replay(const SearchArgs& a, const ReplayArgs& ra, int E, int G, int degw,
                          int blocks, cudaStream_t st, int* occ) {
    switch (E) {
        case 2: return replay_dispatch<2>(a, ra, G, degw, blocks, st, occ);
        case 3: return replay_dispatch<3>(a, ra, G, degw, blocks, st, occ);
        case 5: return replay_dispatch<5>(a, ra, G, degw, blocks, st, occ);
        case 9: return replay_dispatch<9>(a, ra, G, degw, blocks, st, occ);
        case 17: return replay_dispatch<17>(a, ra, G, degw, blocks, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lqg
