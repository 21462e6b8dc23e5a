// Dispatch of the fast search kernel over its pool-size instances.
#include "lqg_internal.h"

namespace lqg {

template <int E>
cudaError_t fast_dispatch(const SearchArgs& a, int G, int degw, int warps, int blocks,
                          size_t smem, cudaStream_t st, int* occ);
extern template cudaError_t fast_dispatch<1>(const SearchArgs&, int, int, int, int, size_t,
                                             cudaStream_t, int*);
extern template cudaError_t fast_dispatch<2>(const SearchArgs&, int, int, int, int, size_t,
                                             cudaStream_t, int*);
extern template cudaError_t fast_dispatch<4>(const SearchArgs&, int, int, int, int, size_t,
                                             cudaStream_t, int*);
extern template cudaError_t fast_dispatch<8>(const SearchArgs&, int, int, int, int, size_t,
                                             cudaStream_t, int*);
extern template cudaError_t fast_dispatch<16>(const SearchArgs&, int, int, int, int, size_t,
                                              cudaStream_t, int*);

size_t fast_smem_bytes(uint32_t dim, uint32_t vbits, int warps) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 8 * dpad + (size_t)warps * (4 * dpad + 4 * ((size_t)1 << vbits) + kCandBytes);
}

static cudaError_t dispatch(const SearchArgs& a, int E, int G, int degw, int warps, int blocks,
                            size_t smem, cudaStream_t st, int* occ) {
    switch (E) {
        case 1: return fast_dispatch<1>(a, G, degw, warps, blocks, smem, st, occ);
        case 2: return fast_dispatch<2>(a, G, degw, warps, blocks, smem, st, occ);
        case 4: return fast_dispatch<4>(a, G, degw, warps, blocks, smem, st, occ);
        case 8: return fast_dispatch<8>(a, G, degw, warps, blocks, smem, st, occ);
        case 16: return fast_dispatch<16>(a, G, degw, warps, blocks, smem, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fast(const SearchArgs& a, int E, int G, int degw, int warps, int blocks,
                        cudaStream_t st) {
    return dispatch(a, E, G, degw, warps, blocks, fast_smem_bytes(a.dim, a.vbits, warps), st,
                    nullptr);
}

int fast_occupancy(int E, int G, int degw, int warps, uint32_t dim, uint32_t vbits) {
    SearchArgs a{};
    a.dim = dim;
    a.vbits = vbits;
    int occ = 0;
    if (dispatch(a, E, G, degw, warps, 0, fast_smem_bytes(dim, vbits, warps), nullptr, &occ) !=
        cudaSuccess)
        return 0;
    return occ;
}

}  // namespace lqg
