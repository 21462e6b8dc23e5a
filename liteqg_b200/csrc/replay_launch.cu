// Dispatch of the replay search kernel over its pool-size instances.
#include "heap_ops.cuh"
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

size_t replay_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t scap, int swarps) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 8 * dpad + (size_t)swarps * replay_warp_bytes(dim, vbits, scap);
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

namespace lqg {

// Result-heap replay pass (qg.hpp:329-343), one warp per query: the logged
// accepted nodes, in order, on a result heap laid out as GCC libstdc++ leaves
// it (heap_ops.cuh: push_heap = sift-up while comp(parent, value); pop_heap =
// hole from the root to a leaf along the larger child, the right one unless
// comp(right, left), then sift-up of the last element). Each push is checked
// against the reference's acceptance test on this heap (size < ef or top >
// distance), and the search warp's bound after it against rp.top(); then the
// output is the first k pops (results[k-1-j] = j-th pop) and, if asked, the
// whole pool in ascending order. The log is read 32 entries per coalesced
// load. A query that fails a check goes to the spill list.
__global__ void __launch_bounds__(256) rp_replay_kernel(SearchArgs a, ReplayArgs ra) {
    using namespace heapops;
    extern __shared__ uint2 hs[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const HeapView rp{hs + (size_t)warp * ra.rcap, nullptr, ra.rcap};
    for (int64_t qi = (int64_t)blockIdx.x * wpb + warp; qi < a.m; qi += (int64_t)gridDim.x * wpb) {
        const uint32_t len = ra.rlen[qi];
        // kNoId: the search failed (already on the spill list); kRlenDone: the
        // search warp wrote the output
        if (len == kNoId || len == kRlenDone) continue;
        if (!replay_result(a, ra, qi, len, rp, lane) && lane == 0) {
            const uint32_t i = atomicAdd(ra.nspill, 1u);
            ra.spill[i] = (int32_t)qi;
        }
        __syncwarp();
    }
}

cudaError_t launch_rp_replay(const SearchArgs& a, const ReplayArgs& ra, cudaStream_t st) {
    if (a.m <= 0) return cudaSuccess;
    constexpr int kWarps = 8;
    const size_t smem = (size_t)ra.rcap * kWarps * sizeof(uint2);
    cudaError_t e = cudaFuncSetAttribute(rp_replay_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t blocks = (a.m + kWarps - 1) / kWarps;
    rp_replay_kernel<<<(unsigned)blocks, kWarps * 32, smem, st>>>(a, ra);
    return cudaGetLastError();
}

}  // namespace lqg
