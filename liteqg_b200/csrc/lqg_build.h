// Internal declarations of the index-build kernels (build_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lqg {

constexpr int kPruneThreads = 128;
constexpr int kCandMax = 256;  // candidates gathered per node
constexpr int kPruneMax = 96;  // nearest candidates that enter the prune
constexpr int kTileD = 128;    // dimensions per shared-memory tile

struct PruneArgs {
    const float* x;  // [n][dim] raw vectors (device)
    uint64_t n;
    uint32_t dim, deg;
    uint64_t node0;  // first node of this launch
    // candidate sources (any may be null)
    const uint32_t* pool;  // [nodes][pool_stride], row 0 = node0
    uint32_t pool_stride, pool_take;
    const uint32_t* nb;      // [n][deg]
    const uint32_t* nb_cnt;  // [n] or null (= deg)
    const uint32_t* rev;        // reverse sources, CSR values
    const uint32_t* rev_start;  // [n] segment start in rev
    const uint32_t* rev_end;    // [n] segment end
    uint32_t rev_cap;           // sources taken per node (lowest ids first)
    // outputs
    uint32_t out_cap;    // ids written per node at most (0 = deg)
    uint32_t* out;       // [n][deg]
    uint32_t* out_cnt;   // [n] ids written
    uint32_t* kept_cnt;  // [n] ids kept by the prune (or null)
    int fill;            // pad with this launch's pruned candidates
    const uint32_t* rest_fill;  // then with an earlier launch's pruned list
    const uint32_t* rest_fill_cnt;
    uint32_t* rest;  // [n][rest_stride] pruned candidates, ascending (or null)
    uint32_t* rest_cnt;
    uint32_t rest_stride;
    float alpha2;  // occlusion factor squared (squared distances): prune i if
                   // alpha2 * d(j, i) < d(node, i); 1 = heuristic_prune
    // search-path candidates (index build): [nodes][path_stride] popped ids,
    // row 0 = node0; up to far_take of them beyond the nearest
    // kPruneMax - far_take candidates also enter the prune
    const uint32_t* path;
    uint32_t path_stride, path_take, far_take;
    // slots of a list that only candidates farther than 4x the nearest
    // candidate's squared distance may take (long links)
    uint32_t far_budget;
    // candidate-to-candidate distances: 0 FP32 on the CUDA cores; 1 BF16 Gram
    // matrices on the tensor cores (tcgen05) with FP32 re-checks of the
    // decisions near their threshold
    int pair_tc;
    uint32_t* err;                   // bit 0: a tensor-core wait timed out
    unsigned long long* rechecks;    // FP32 re-checks made (or null)
};

cudaError_t launch_sq8_encode(const float* x, uint64_t n, uint32_t dim, float* params,
                              uint8_t* codes, float* work, cudaStream_t st);
size_t sq8_work_floats(uint32_t dim);
cudaError_t launch_entry(const float* x, uint64_t n, uint32_t dim, double* work, float* centroid,
                         unsigned long long* best, cudaStream_t st);
size_t entry_work_doubles(uint32_t dim);
cudaError_t launch_random_fill(uint32_t* out, const uint32_t* from, uint64_t n, uint32_t deg,
                               uint64_t seed, cudaStream_t st);
cudaError_t launch_prune(const PruneArgs& a, uint64_t nodes, cudaStream_t st);
struct ReverseWork {
    uint32_t *keys_in, *vals_in, *keys_out, *vals_out;  // [n * deg] each
    uint32_t *start, *end;                              // [n] each
    void* temp;
    size_t temp_bytes;
};
size_t reverse_temp_bytes(uint64_t n, uint32_t deg);
cudaError_t launch_reverse(const uint32_t* nb, const uint32_t* cnt, uint64_t n, uint32_t deg,
                           ReverseWork& w, cudaStream_t st);

}  // namespace lqg
