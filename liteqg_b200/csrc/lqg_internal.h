// Internal host-side declarations shared by the kernels file and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lqg_kernels.cuh"

namespace lqg {

// One persistent launch of the fast kernel (E pool registers per lane,
// G lanes per candidate, degw = degree_bound / 32).
cudaError_t launch_fast(const SearchArgs& a, int E, int G, int degw, int warps, int blocks,
                        cudaStream_t st);
// Resident blocks per SM for that instance (0 if it cannot launch).
int fast_occupancy(int E, int G, int degw, int warps, uint32_t dim, uint32_t vbits);
size_t fast_smem_bytes(uint32_t dim, uint32_t vbits, int warps);

// One launch of the exact kernel over a work list; blocks*warps must equal
// the number of scratch slots in s.
cudaError_t launch_exact(const SearchArgs& a, const ExactScratch& s, int degw, int warps,
                         int blocks, cudaStream_t st);
size_t exact_smem_bytes(uint32_t dim, int warps);

// Heap kernel: per-warp shared-memory capacities and the list of queries whose
// search pool outgrew them (handed to the exact kernel).
struct HeapArgs {
    uint32_t rcap;       // result-pool slots (>= ef + 1), shared memory
    uint32_t scap;       // search-pool slots in shared memory
    uint2* sp_global;    // [warps][gcap] further search-pool slots
    uint32_t gcap;
    int32_t* spill;      // [m] queries whose search pool outgrew scap + gcap
    uint32_t* nspill;
};

__host__ __device__ inline size_t heap_warp_bytes(uint32_t dim, uint32_t vbits, uint32_t rcap,
                                                  uint32_t scap) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 4 * dpad + 4 * ((size_t)1 << vbits) + kCandBytes + 8 * (size_t)rcap + 8 * (size_t)scap;
}
size_t heap_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t rcap, uint32_t scap, int warps);
// Launches the heap kernel (or, with occ != null, only reports resident blocks per SM).
cudaError_t launch_heap(const SearchArgs& a, const HeapArgs& h, int G, int degw, int warps,
                        int blocks, cudaStream_t st, int* occ);

// Replay kernel (replay_kernel.cuh): sorted-pool search warps plus one
// search-heap replay warp per block, then a result-heap replay pass (one
// thread per query). E = replay_pool_regs(ef_max) (0: ef too large).
struct ReplayArgs {
    uint32_t swarps;     // search warps per block (the replay warp follows)
    uint32_t scap;       // search-heap slots in shared memory
    uint2* sp_global;    // [blocks * swarps][gcap] further search-heap slots
    uint32_t gcap;
    int32_t* spill;      // queries handed to the exact kernel
    uint32_t* nspill;
    uint4* rlog;         // [m][rlog_cap] (id, distance, bound after, 0) per accepted node
    uint32_t rlog_cap;
    uint32_t* rlen;      // [m] accepted nodes logged, 0xFFFFFFFF if the search failed
    uint32_t rcap;       // result-heap slots (>= ef + 1) of the replay pass
    uint32_t efcap;      // largest ef: min(sorted-pool slots - 32, rcap - 1)
    uint32_t replay_all; // split/batch kernels: replay every query's result heap (else
                         // only those whose output the heap layout decides)
    uint32_t acap;       // batch kernel: sorted-pool slots (>= efcap + 32)
    uint32_t lazy;       // batch kernel: build the search heap only at the first tied pop
    uint2* plog;         // [m][rlog_cap] (accepted before the pop, popped id) per pop
};
constexpr uint32_t kRlenDone = 0xFFFFFFFEu;  // rlen: output already written
constexpr uint32_t kReplayLogN = 128;  // search-heap log ring entries (8 bytes) per search warp

// Shared memory of one search warp: query, visited cache, candidates, log
// ring, search heap, control words.
__host__ __device__ inline size_t replay_warp_bytes(uint32_t dim, uint32_t vbits, uint32_t scap) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 4 * dpad + 4 * ((size_t)1 << vbits) + kCandBytes + 8 * (size_t)kReplayLogN +
           8 * (size_t)scap + 16;
}
int replay_pool_regs(uint32_t ef_max);
size_t replay_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t scap, int swarps);
cudaError_t launch_replay(const SearchArgs& a, const ReplayArgs& ra, int E, int G, int degw,
                          int blocks, cudaStream_t st, int* occ);
// Split kernel (split_kernel.cuh): exact search heap per warp, sorted
// register array for the bound, result log for the replay pass.
size_t split_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t scap, int warps);
bool split_replays_in_place_host(uint32_t vbits, uint32_t scap, uint32_t rcap);
cudaError_t launch_split(const SearchArgs& a, const ReplayArgs& ra, int E, int G, int degw,
                         int warps, int blocks, cudaStream_t st, int* occ);
// Batched-acceptance kernel (batch_kernel.cuh): exact search heap per warp,
// sorted pool in shared memory, each expansion's candidates decided at once.
size_t batch_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t scap, uint32_t acap, int warps);
bool batch_replays_in_place_host(uint32_t vbits, uint32_t scap, uint32_t acap, uint32_t rcap);
cudaError_t launch_batch(const SearchArgs& a, const ReplayArgs& ra, int G, int degw, int warps,
                         int blocks, cudaStream_t st, int* occ);
// Its query-per-block form (batch_cta.cu): one query per block of 4 warps,
// each expansion's distances split over the warps; for batches smaller than
// the GPU's resident warps, where a query's latency sets the batch time.
cudaError_t launch_batch_cta(const SearchArgs& a, const ReplayArgs& ra, int degw, int blocks,
                             cudaStream_t st, int* occ);
// Result-heap replay pass over a[0, m): one warp per query.
cudaError_t launch_rp_replay(const SearchArgs& a, const ReplayArgs& ra, cudaStream_t st);

}  // namespace lqg
