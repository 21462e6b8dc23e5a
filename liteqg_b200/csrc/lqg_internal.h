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

}  // namespace lqg
