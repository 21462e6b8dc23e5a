// Index-build kernels: SQ8 encoding, entry point, random initial graph, and
// the candidate pruning that turns search pools into neighbour lists.
//
// Reference: QGBuilder (symqglib/qg/qg_builder.hpp:48-376),
// sq8_quantize (symqglib/quantization/sq8.hpp:11-26), compute_centroid /
// exact_nn (symqglib/space/space.hpp:16-78).
//
// The SQ8 encoder reproduces the reference's file contents exactly (the codes
// and parameters of a reference-built index are pinned by the tests): per-dim
// min/max, scale = (max - min) * (1/255) — the reference's -Ofast build turns
// its division by the constant 255 into that multiply — and
// code = round_half_away((v - min) / scale) with a true division.
//
// Pruning follows heuristic_prune (qg_builder.hpp:155-200): candidates in
// ascending exact distance; a candidate is kept unless an already-kept one
// lies closer to it than the node does (d(kept, c) < d(node, c)); with an
// occlusion factor alpha > 1 (squared distances: alpha^2 d(kept, c) <
// d(node, c)) the longer links of the Vamana rule survive too.
// The candidate-to-candidate distances of one node form a P x P matrix that
// one CTA accumulates in registers over 128-dimension tiles staged in shared
// memory.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <math_constants.h>

#include <cub/device/device_radix_sort.cuh>

#include "lqg_build.h"

namespace lqg {

// ---- SQ8 encode ---------------------------------------------------------
//
// The per-dimension min and max follow std::min / std::max over the rows in
// order (quantization/sq8.hpp:13-17) as the reference's -Ofast build compiles
// them (minss/maxss, new value second): a value replaces the running one
// unless that one is strictly smaller (larger), so among equal values the
// last row's is kept. That decides the sign of a zero minimum (-0.0 and 0.0
// compare equal) and so the file's bytes. Each block folds its rows in order,
// then the blocks' results are folded in order; the fold keeps the last of
// the equal values, so it does not depend on where the blocks split.

__global__ void minmax_partial_kernel(const float* __restrict__ x, uint64_t n, uint32_t dim,
                                      uint64_t rows_per_block, float* __restrict__ pmin,
                                      float* __restrict__ pmax) {
    const uint64_t r0 = (uint64_t)blockIdx.x * rows_per_block;
    const uint64_t r1 = min(n, r0 + rows_per_block);
    for (uint32_t d = threadIdx.x; d < dim; d += blockDim.x) {
        float mn = CUDART_INF_F, mx = -CUDART_INF_F;
        if (r0 < r1) mn = mx = x[r0 * dim + d];
        for (uint64_t i = r0 + 1; i < r1; ++i) {
            const float v = x[i * dim + d];
            mn = mn < v ? mn : v;
            mx = mx > v ? mx : v;
        }
        pmin[(size_t)blockIdx.x * dim + d] = mn;
        pmax[(size_t)blockIdx.x * dim + d] = mx;
    }
}

__global__ void minmax_final_kernel(const float* __restrict__ pmin, const float* __restrict__ pmax,
                                    uint32_t nblocks, uint32_t dim, float* __restrict__ params) {
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < dim; d += gridDim.x * blockDim.x) {
        float mn = pmin[d], mx = pmax[d];
        for (uint32_t b = 1; b < nblocks; ++b) {
            const float lo = pmin[(size_t)b * dim + d], hi = pmax[(size_t)b * dim + d];
            mn = mn < lo ? mn : lo;
            mx = mx > hi ? mx : hi;
        }
        params[2 * d] = mn;
        params[2 * d + 1] = __fmul_rn(__fsub_rn(mx, mn), 1.0f / 255.0f);
    }
}

__global__ void sq8_encode_kernel(const float* __restrict__ x, uint64_t total, uint32_t dim,
                                  const float* __restrict__ params, uint8_t* __restrict__ codes) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t d = (uint32_t)(e % dim);
        const float mn = params[2 * d], sc = params[2 * d + 1];
        uint8_t c = 0;
        if (sc > 0.f) {
            const float q = roundf(__fdiv_rn(__fsub_rn(x[e], mn), sc));
            c = (uint8_t)fminf(fmaxf(q, 0.f), 255.f);
        }
        codes[e] = c;
    }
}

// ---- entry point ----------------------------------------------------------

__global__ void centroid_partial_kernel(const float* __restrict__ x, uint64_t n, uint32_t dim,
                                        uint64_t rows_per_block, double* __restrict__ part) {
    const uint64_t r0 = (uint64_t)blockIdx.x * rows_per_block;
    const uint64_t r1 = min(n, r0 + rows_per_block);
    for (uint32_t d = threadIdx.x; d < dim; d += blockDim.x) {
        double s = 0.0;
        for (uint64_t i = r0; i < r1; ++i) s += (double)x[i * dim + d];
        part[(size_t)blockIdx.x * dim + d] = s;
    }
}

__global__ void centroid_final_kernel(const double* __restrict__ part, uint32_t nblocks,
                                      uint32_t dim, uint64_t n, float* __restrict__ centroid) {
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < dim; d += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint32_t b = 0; b < nblocks; ++b) s += part[(size_t)b * dim + d];
        centroid[d] = (float)(s * (1.0 / (double)n));
    }
}

// Squared L2 of two float vectors in the reference's 16-lane order (l2.hpp).
__device__ __forceinline__ float l2_ref_order(const float* a, const float* b, uint32_t dim) {
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) acc[l] = 0.f;
    const uint32_t mul = dim & ~15u;
    for (uint32_t d = 0; d < mul; d += 16) {
#pragma unroll
        for (int l = 0; l < 16; ++l) {
            const float t = __fsub_rn(a[d + l], b[d + l]);
            acc[l] = __fmaf_rn(t, t, acc[l]);
        }
    }
#pragma unroll
    for (int h = 8; h >= 1; h >>= 1)
#pragma unroll
        for (int l = 0; l < h; ++l) acc[l] = __fadd_rn(acc[l], acc[l + h]);
    float r = acc[0];
    for (uint32_t d = mul; d < dim; ++d) {
        const float t = __fsub_rn(a[d], b[d]);
        r = __fmaf_rn(t, t, r);
    }
    return r;
}

// l2_ref_order for 16-byte aligned rows (dimension a multiple of 4): the same
// operations in the same order, read four floats per load.
__device__ __forceinline__ float l2_ref_order_v4(const float* a, const float* b, uint32_t dim) {
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) acc[l] = 0.f;
    const uint32_t mul = dim & ~15u;
    const float4* a4 = reinterpret_cast<const float4*>(a);
    const float4* b4 = reinterpret_cast<const float4*>(b);
#pragma unroll 2
    for (uint32_t d = 0; d < mul; d += 16) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 x = a4[d / 4 + q], y = __ldg(b4 + d / 4 + q);
            float t;
            t = __fsub_rn(x.x, y.x); acc[4 * q + 0] = __fmaf_rn(t, t, acc[4 * q + 0]);
            t = __fsub_rn(x.y, y.y); acc[4 * q + 1] = __fmaf_rn(t, t, acc[4 * q + 1]);
            t = __fsub_rn(x.z, y.z); acc[4 * q + 2] = __fmaf_rn(t, t, acc[4 * q + 2]);
            t = __fsub_rn(x.w, y.w); acc[4 * q + 3] = __fmaf_rn(t, t, acc[4 * q + 3]);
        }
    }
#pragma unroll
    for (int h = 8; h >= 1; h >>= 1)
#pragma unroll
        for (int l = 0; l < h; ++l) acc[l] = __fadd_rn(acc[l], acc[l + h]);
    float r = acc[0];
    for (uint32_t d = mul; d < dim; ++d) {
        const float t = __fsub_rn(a[d], b[d]);
        r = __fmaf_rn(t, t, r);
    }
    return r;
}

// exact_nn (space.hpp:16-48): argmin over all points of l2(x_i, centroid);
// ties go to the smallest id. best = (distance bits << 32) | id.
__global__ void nearest_kernel(const float* __restrict__ x, uint64_t n, uint32_t dim,
                               const float* __restrict__ centroid,
                               unsigned long long* __restrict__ best) {
    unsigned long long mine = ~0ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float d = l2_ref_order(x + i * dim, centroid, dim);
        const unsigned long long key = ((unsigned long long)__float_as_uint(d) << 32) | i;
        mine = key < mine ? key : mine;
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long v = __shfl_down_sync(0xFFFFFFFFu, mine, o);
        mine = v < mine ? v : mine;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(best, mine);
}

// ---- random initial graph (qg_builder.hpp:263-291) -------------------------

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint32_t rand_id(uint64_t seed, uint64_t node, uint32_t j,
                                            uint32_t attempt, uint64_t n) {
    const uint64_t h = mix64(seed ^ mix64(node * 0x100000001B3ull + j * 7919u + attempt * 104729u));
    return (uint32_t)(h % n);
}

// Fills out[node][from..deg) with distinct random ids, none equal to node or
// to out[node][0..from). One warp per node; n > deg is required.
__global__ void random_fill_kernel(uint32_t* __restrict__ out, const uint32_t* __restrict__ from,
                                   uint64_t n, uint32_t deg, uint64_t seed) {
    const uint64_t node = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (node >= n) return;
    uint32_t* row = out + node * deg;
    const uint32_t f = from ? min(from[node], deg) : 0u;
    uint32_t filled = f;
    uint32_t attempt = 0;
    while (filled < deg && attempt < 4096) {
        const uint32_t want = deg - filled;
        uint32_t c = rand_id(seed, node, lane, attempt++, n);
        bool ok = lane < (int)want && c != (uint32_t)node;
        for (uint32_t j = 0; j < filled; ++j) ok = ok && row[j] != c;
        const unsigned mm = __match_any_sync(0xFFFFFFFFu, ok ? c : 0xFFFFFFFFu);
        uint32_t lt;
        asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
        ok = ok && (mm & lt) == 0;
        const unsigned b = __ballot_sync(0xFFFFFFFFu, ok);
        if (ok) row[filled + __popc(b & lt)] = c;
        filled += __popc(b);
        __syncwarp();
    }
    // Bounded fallback (n > deg guarantees it completes): the next ids after
    // the node, skipping the node and ids already present.
    if (lane == 0) {
        for (uint64_t t = 1; filled < deg && t < n; ++t) {
            const uint32_t c = (uint32_t)((node + t) % n);
            bool dup = false;
            for (uint32_t j = 0; j < filled && !dup; ++j) dup = row[j] == c;
            if (!dup) row[filled++] = c;
        }
    }
    __syncwarp();
}

// ---- candidate-to-candidate distances on the tensor cores (tcgen05) -------
//
// The prune's P x P matrix of squared distances among a node's candidates
// (P <= 96) as one BF16 Gram matrix per 128-dimension chunk, accumulated in
// FP32 in tensor memory: rows are the candidates minus the node's vector
// (so norms are on the scale of the distances), rounded to BF16 and staged in
// shared memory in the canonical K-major layout without swizzle (8-row x
// 16-byte core matrices; the 16 core matrices of a row group's 128 dimensions
// are 128 bytes apart (LBO), row groups 2048 bytes apart (SBO)). One thread
// issues tcgen05.mma.cta_group::1.kind::f16 with M = 128 (rows past P are
// zero), N = 96, K = 16 per instruction; the result is read back with
// tcgen05.ld (warp w owns tensor-memory lanes 32w..32w+31) and
// d~(i, j) = n~i + n~j - 2 G(i, j) with n~ the norms of the rounded rows.
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (sm_100): start address, leading and
// stride byte offsets (all >> 4), version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::f16: BF16 A and B (K-major), FP32 D.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t m, uint32_t n) {
    return (1u << 4)            // D format F32
           | (1u << 7)          // A format BF16
           | (1u << 10)         // B format BF16
           | ((n >> 3) << 17)   // N / 8
           | ((m >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u),
          "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// Bounded wait for the mbarrier phase with this parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
    const uint32_t a = smem_u32(mbar);
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc

// ---- candidate pruning ---------------------------------------------------

// One CTA (kPruneThreads) per node.
//  1. Gather candidates from up to three sources (pool rows, neighbour rows
//     with counts, reverse rows with counts); drop the node and duplicates.
//  2. Exact FP32 distance node -> candidate (reference 16-lane order).
//  3. Sort ascending (bitonic, kCandMax), keep the nearest kPruneMax.
//  4. Candidate-to-candidate distances, then the greedy RNG prune.
//  5. Write up to deg kept ids; with fill, pad to exactly deg with the pruned
//     candidates in distance order (the spirit of graph_refine,
//     qg_builder.hpp:293-348) and mark the row count; rest rows receive the
//     pruned candidates for a later fill.
// TC selects the candidate-to-candidate distance form at compile time (1:
// BF16 Gram matrices on the tensor cores, 0: FP32 on the CUDA cores), so
// each instance holds only its own path's registers.
template <int TC>
__global__ void __launch_bounds__(kPruneThreads) prune_kernel(PruneArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_ids[kCandMax];
    __shared__ float s_d[kCandMax];
    __shared__ uint32_t s_cnt;
    __shared__ uint8_t s_keep[kPruneMax];   // 1 kept
    // FP32 path: tile [kPruneMax+1][kTileD+1] floats; tensor-core path: the
    // BF16 hi and lo operands, 128 rows x kTileD each; then pair
    // [kPruneMax][kPruneMax]
    float* tile = reinterpret_cast<float*>(smem);
    float* pair = tile + (TC ? 128 * kTileD : (kPruneMax + 1) * (kTileD + 1));

    const uint64_t node = blockIdx.x + a.node0;
    if (node >= a.n) return;
    const int tid = threadIdx.x;
    const uint32_t dim = a.dim;
    if (tid == 0) s_cnt = 0;
    for (int i = tid; i < kCandMax; i += kPruneThreads) {
        s_ids[i] = 0xFFFFFFFFu;
        s_d[i] = CUDART_INF_F;
    }
    __syncthreads();

    // 1. gather into fixed slots, source after source, up to kCandMax (so the
    // candidate set does not depend on thread timing); duplicates removed
    // below after sorting by id. Entries are id << 1 | from_path (ids < 2^31);
    // the node itself and out-of-range ids become empty slots.
    auto put = [&](uint32_t slot, uint32_t v, uint32_t from_path) {
        s_ids[slot] = (v == (uint32_t)node || v >= a.n) ? 0xFFFFFFFFu : ((v << 1) | from_path);
    };
    uint32_t off = 0;
    if (a.pool) {
        const uint32_t* p = a.pool + (node - a.node0) * a.pool_stride;
        const uint32_t c = min(a.pool_take, (uint32_t)kCandMax - off);
        for (uint32_t j = tid; j < c; j += kPruneThreads) put(off + j, p[j], 0u);
        off += c;
    }
    if (a.path) {
        const uint32_t* p = a.path + (node - a.node0) * a.path_stride;
        const uint32_t c = min(a.path_take, (uint32_t)kCandMax - off);
        for (uint32_t j = tid; j < c; j += kPruneThreads) put(off + j, p[j], 1u);
        off += c;
    }
    if (a.nb) {
        const uint32_t c = min(a.nb_cnt ? min(a.nb_cnt[node], a.deg) : a.deg, (uint32_t)kCandMax - off);
        for (uint32_t j = tid; j < c; j += kPruneThreads) put(off + j, a.nb[node * a.deg + j], 0u);
        off += c;
    }
    if (a.rev) {
        const uint32_t s0 = a.rev_start[node], s1 = a.rev_end[node];
        const uint32_t c = min(min(s1 - s0, a.rev_cap), (uint32_t)kCandMax - off);
        for (uint32_t j = tid; j < c; j += kPruneThreads) put(off + j, a.rev[s0 + j], 0u);
        off += c;
    }
    __syncthreads();
    const uint32_t cnt = off;

    // 2. exact distances node -> candidate (ids first sorted to drop dups)
    // bitonic sort by id to find duplicates
    for (uint32_t k = 2; k <= kCandMax; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = tid; i < kCandMax; i += kPruneThreads) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const uint32_t x = s_ids[i], y = s_ids[l];
                    if ((x > y) == up) {
                        s_ids[i] = y;
                        s_ids[l] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    const float* xn = a.x + node * dim;
    // rows start on 16-byte boundaries: four floats per load
    const bool v4 = (dim & 3u) == 0 && (reinterpret_cast<uintptr_t>(a.x) & 15u) == 0;
    for (uint32_t i = tid; i < cnt; i += kPruneThreads) {
        const uint32_t v = s_ids[i];
        // keep the last of equal ids (the path-flagged copy, if any)
        const bool dup = i + 1 < cnt && (s_ids[i + 1] >> 1) == (v >> 1);
        const float* xv = a.x + (uint64_t)(v >> 1) * dim;
        s_d[i] = (dup || v == 0xFFFFFFFFu) ? CUDART_INF_F
                 : v4                      ? l2_ref_order_v4(xn, xv, dim)
                                           : l2_ref_order(xn, xv, dim);
    }
    __syncthreads();
    // 3. sort ascending by (distance, id)
    for (uint32_t k = 2; k <= kCandMax; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = tid; i < kCandMax; i += kPruneThreads) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const float dx = s_d[i], dy = s_d[l];
                    const uint32_t ix = s_ids[i], iy = s_ids[l];
                    const bool gt = dx > dy || (dx == dy && ix > iy);
                    if (gt == up) {
                        s_d[i] = dy;
                        s_d[l] = dx;
                        s_ids[i] = iy;
                        s_ids[l] = ix;
                    }
                }
            }
            __syncthreads();
        }
    }
    uint32_t P = 0;
    {
        // valid candidates are the finite-distance prefix
        __shared__ uint32_t s_valid;
        if (tid == 0) s_valid = 0;
        __syncthreads();
        for (uint32_t i = tid; i < kCandMax; i += kPruneThreads)
            if (s_d[i] < CUDART_INF_F) atomicAdd(&s_valid, 1u);
        __syncthreads();
        const uint32_t V = s_valid;
        if (a.path && a.far_take && V > (uint32_t)kPruneMax) {
            // the nearest kPruneMax - far_take, then search-path candidates
            // beyond them in distance order; compacted in place
            if (tid == 0) {
                const uint32_t near = kPruneMax - min(a.far_take, (uint32_t)kPruneMax);
                uint32_t w = near, taken = 0;
                for (uint32_t i = near; i < V && taken < a.far_take; ++i)
                    if (s_ids[i] & 1u) {
                        s_ids[w] = s_ids[i];
                        s_d[w] = s_d[i];
                        ++w;
                        ++taken;
                    }
                s_valid = w;
            }
            __syncthreads();
            P = s_valid;
        } else {
            P = min(V, (uint32_t)kPruneMax);
        }
    }

    // 4. pairwise distances among the first P candidates
    __shared__ uint64_t s_mbar;
    __shared__ uint32_t s_tmem;
    __shared__ float s_norm[128];
    __shared__ int s_exact;
    if (tid == 0) s_exact = 0;
    if constexpr (TC != 0) {
        // Gram matrices on the tensor cores (see tc:: above), each centred
        // value split into BF16 hi + lo (x = hi + lo + r, |r| <= 2^-16 |x|):
        // G~ = Ghh + Ghl + Ghl^T, two accumulators in tensor memory (columns
        // 0.. and 128..), so the BF16 error that decides how many decisions
        // need an FP32 re-check is 2^-16 instead of 2^-8.
        __nv_bfloat16* op_hi = reinterpret_cast<__nv_bfloat16*>(tile);  // 128 x 128, 32 KB
        __nv_bfloat16* op_lo = op_hi + 128 * kTileD;                      // 128 x 128, 32 KB
        if (tid < 32) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                         ::"r"(tc::smem_u32(&s_tmem)), "r"(256u));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
        if (tid == 0) {
            tc::mbar_init(&s_mbar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = s_tmem;
        const float* xn = a.x + node * dim;
        const float* xr = a.x + (uint64_t)(s_ids[tid < P ? tid : 0] >> 1) * dim;
        float nrm = 0.f;  // |hi|^2 + 2 hi.lo: the Gram diagonal's form
        bool ok = true, rounded = false;
        uint32_t chunk = 0;
        for (uint32_t d0 = 0; d0 < dim; d0 += kTileD, ++chunk) {
            // row tid of this chunk: x_candidate - x_node split, zero past P and dim
#pragma unroll 2
            for (uint32_t kc = 0; kc < kTileD / 8; ++kc) {
                uint32_t wh[4], wl[4];
                float f[8];
                const uint32_t db = d0 + kc * 8;
                if (v4 && tid < P && db + 8 <= dim) {
                    const float4 r0 = __ldg(reinterpret_cast<const float4*>(xr + db));
                    const float4 r1 = __ldg(reinterpret_cast<const float4*>(xr + db + 4));
                    const float4 n0 = __ldg(reinterpret_cast<const float4*>(xn + db));
                    const float4 n1 = __ldg(reinterpret_cast<const float4*>(xn + db + 4));
                    f[0] = __fsub_rn(r0.x, n0.x); f[1] = __fsub_rn(r0.y, n0.y);
                    f[2] = __fsub_rn(r0.z, n0.z); f[3] = __fsub_rn(r0.w, n0.w);
                    f[4] = __fsub_rn(r1.x, n1.x); f[5] = __fsub_rn(r1.y, n1.y);
                    f[6] = __fsub_rn(r1.z, n1.z); f[7] = __fsub_rn(r1.w, n1.w);
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        f[e] = tid < P && db + e < dim ? __fsub_rn(xr[db + e], xn[db + e]) : 0.f;
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float f0 = f[2 * e], f1 = f[2 * e + 1];
                    const __nv_bfloat162 h = __floats2bfloat162_rn(f0, f1);
                    const float h0 = __low2float(h), h1 = __high2float(h);
                    // f - hi is exact in FP32 (at most 16 significant bits)
                    const __nv_bfloat162 l =
                        __floats2bfloat162_rn(__fsub_rn(f0, h0), __fsub_rn(f1, h1));
                    const float l0 = __low2float(l), l1 = __high2float(l);
                    rounded |= h0 != f0 || h1 != f1;
                    nrm = __fmaf_rn(h0, h0, nrm);
                    nrm = __fmaf_rn(2.f * h0, l0, nrm);
                    nrm = __fmaf_rn(h1, h1, nrm);
                    nrm = __fmaf_rn(2.f * h1, l1, nrm);
                    wh[e] = *reinterpret_cast<const uint32_t*>(&h);
                    wl[e] = *reinterpret_cast<const uint32_t*>(&l);
                }
                const uint32_t off = kc * 128 + (tid >> 3) * 2048 + (tid & 7) * 16;
                *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(op_hi) + off) =
                    make_uint4(wh[0], wh[1], wh[2], wh[3]);
                *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(op_lo) + off) =
                    make_uint4(wl[0], wl[1], wl[2], wl[3]);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t bh = tc::smem_u32(op_hi), bl = tc::smem_u32(op_lo);
                constexpr uint32_t idesc = tc::idesc_bf16_f32(128, kPruneMax);
#pragma unroll
                for (uint32_t s = 0; s < kTileD / 16; ++s) {
                    const uint64_t dh = tc::smem_desc(bh + s * 256, 128, 2048);
                    const uint64_t dl = tc::smem_desc(bl + s * 256, 128, 2048);
                    const uint32_t acc = (chunk > 0 || s > 0) ? 1u : 0u;
                    tc::mma_bf16(tmem, dh, dh, idesc, acc);          // Ghh
                    tc::mma_bf16(tmem + 128u, dh, dl, idesc, acc);   // Ghl
                }
                tc::commit(&s_mbar);
            }
            // the operand tiles are rewritten next chunk: wait for these MMAs
            if (!tc::mbar_wait(&s_mbar, chunk & 1u)) ok = false;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        s_norm[tid] = nrm;
        // every staged value exact in BF16 and every norm below 2^23: the
        // Gram matrix (its partial sums are bounded by the norms) and the
        // distances are exact, so no decision needs a re-check
        const int exact = !__syncthreads_or(rounded || nrm >= 8388608.0f);
        if (tid == 0) s_exact = exact;
        // row tid of Ghl into the pair buffer, for its transpose
        const uint32_t w = tid >> 5;
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < (uint32_t)kPruneMax; c0 += 16) {
            float g[16];
            tc::ld16(tmem + ((32u * w) << 16) + 128u + c0, g);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (tid < P)
#pragma unroll
                for (int e = 0; e < 16; ++e) pair[tid * kPruneMax + c0 + e] = g[e];
        }
        __syncthreads();
        // squared distances of row tid to the later columns: the upper
        // triangle is rewritten while only the lower one is read
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < (uint32_t)kPruneMax; c0 += 16) {
            float gh[16], gl[16];
            tc::ld16(tmem + ((32u * w) << 16) + c0, gh);
            tc::ld16(tmem + ((32u * w) << 16) + 128u + c0, gl);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (tid < P) {
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const uint32_t c = c0 + e;
                    if (c < P && c > tid) {
                        const float gt = __fadd_rn(__fadd_rn(gh[e], gl[e]), pair[c * kPruneMax + tid]);
                        pair[tid * kPruneMax + c] =
                            fmaxf(0.f, __fsub_rn(__fadd_rn(nrm, s_norm[c]), 2.f * gt));
                    }
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid < 32) {
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u));
        }
        if (!ok && tid == 0 && a.err) atomicOr(a.err, 1u);
    } else {
        if (tid < 128) s_norm[tid] = 0.f;
        // 4. pairwise distances among the first P candidates, tiled over dims.
        // Thread t owns pairs p = t + kPruneThreads * s of the strict upper
        // triangle in row-major order.
        constexpr int kPairsPerThread = (kPruneMax * (kPruneMax - 1) / 2 + kPruneThreads - 1) / kPruneThreads;
        float acc[kPairsPerThread];
        uint32_t pab[kPairsPerThread];  // row | col << 16
        const uint32_t npairs = P * (P - (P > 0 ? 1 : 0)) / 2;
    #pragma unroll
        for (int s = 0; s < kPairsPerThread; ++s) {
            acc[s] = 0.f;
            const uint32_t p = tid + kPruneThreads * s;
            // invert p -> (r, c), r < c, row-major over the upper triangle of P
            uint32_t r = 0, c = 0;
            if (p < npairs) {
                uint32_t rem = p;
                uint32_t rowlen = P - 1;
                while (rem >= rowlen) {
                    rem -= rowlen;
                    ++r;
                    --rowlen;
                }
                c = r + 1 + rem;
            }
            pab[s] = r | (c << 16);
        }
        for (uint32_t d0 = 0; d0 < dim; d0 += kTileD) {
            const uint32_t td = min((uint32_t)kTileD, dim - d0);
            __syncthreads();
            for (uint32_t e = tid; e < P * td; e += kPruneThreads) {
                const uint32_t r = e / td, c = e % td;
                tile[r * (kTileD + 1) + c] = a.x[(uint64_t)(s_ids[r] >> 1) * dim + d0 + c];
            }
            __syncthreads();
    #pragma unroll
            for (int s = 0; s < kPairsPerThread; ++s) {
                const uint32_t p = tid + kPruneThreads * s;
                if (p < npairs) {
                    const float* ra = tile + (pab[s] & 0xFFFFu) * (kTileD + 1);
                    const float* rb = tile + (pab[s] >> 16) * (kTileD + 1);
                    float t = acc[s];
                    for (uint32_t c = 0; c < td; ++c) {
                        const float df = ra[c] - rb[c];
                        t = fmaf(df, df, t);
                    }
                    acc[s] = t;
                }
            }
        }
    #pragma unroll
        for (int s = 0; s < kPairsPerThread; ++s) {
            const uint32_t p = tid + kPruneThreads * s;
            if (p < npairs) pair[(pab[s] & 0xFFFFu) * kPruneMax + (pab[s] >> 16)] = acc[s];
        }
    }
    // 5a. every pair's occlusion decision at once: kept j would prune later i
    // when alpha^2 d(j, i) < d(node, i). On the tensor-core path the split-
    // BF16 estimate decides unless it lies within its error bound of the
    // threshold; then the FP32 value, in the same order as the CUDA-core path,
    // decides. A decision does not depend on which candidates the greedy pass
    // keeps, so all pairs are decided in parallel, one bit each, with no
    // barrier per kept neighbour (the narrow bound leaves few re-checks, and
    // they run spread over the whole block).
    constexpr uint32_t kOccW = (kPruneMax + 31) / 32;
    constexpr uint32_t kRecheckCap = 1024;  // uncertain pairs listed per node
    __shared__ uint32_t s_occ[kPruneMax][kOccW];
    __shared__ uint16_t s_rl[kRecheckCap];   // (j << 7 | i) of uncertain pairs
    __shared__ uint32_t s_nrl;
    for (uint32_t i = tid; i < (uint32_t)kPruneMax * kOccW; i += kPruneThreads)
        (&s_occ[0][0])[i] = 0;
    for (uint32_t i = tid; i < kPruneMax; i += kPruneThreads) s_keep[i] = 0;
    if (tid == 0) s_nrl = 0;
    __syncthreads();
    // the FP32 value of pair (j, i), in the CUDA-core path's order
    auto fp32_pair = [&](uint32_t j, uint32_t i) {
        const float* xj = a.x + (uint64_t)(s_ids[j] >> 1) * dim;
        const float* xi = a.x + (uint64_t)(s_ids[i] >> 1) * dim;
        float t = 0.f;
        uint32_t d = 0;
        if (v4)
            for (; d < dim; d += 4) {
                const float4 p = __ldg(reinterpret_cast<const float4*>(xj + d));
                const float4 q = __ldg(reinterpret_cast<const float4*>(xi + d));
                float df = p.x - q.x;
                t = fmaf(df, df, t);
                df = p.y - q.y;
                t = fmaf(df, df, t);
                df = p.z - q.z;
                t = fmaf(df, df, t);
                df = p.w - q.w;
                t = fmaf(df, df, t);
            }
        for (; d < dim; ++d) {
            const float df = xj[d] - xi[d];
            t = fmaf(df, df, t);
        }
        return t;
    };
    for (uint32_t e = tid; e < P * P; e += kPruneThreads) {
        const uint32_t j = e / P, i = e % P;
        if (i <= j) continue;
        float dji = pair[j * kPruneMax + i];
        if (TC && !s_exact) {
            // bound on |estimate - FP32 value|: the split's residuals
            // (2^-15 sqrt(d) (|a| + |b|)), the missing lo.lo term
            // (2^-15 (na + nb)), FP32 accumulation in tensor memory and in the
            // FP32 path (about 2 D 2^-24 (na + nb) each), with a factor of 2 to spare
            const float ni = s_norm[i], nj = s_norm[j];
            const float err = 6.103515625e-05f * sqrtf(fmaxf(dji, 0.f)) * (sqrtf(ni) + sqrtf(nj)) +
                              (2.384185791015625e-07f * (float)dim + 1.220703125e-04f) * (ni + nj);
            if (fabsf(a.alpha2 * dji - s_d[i]) <= a.alpha2 * err) {
                // listed, and re-checked below by all threads at once (a
                // re-check in this loop would keep its warp's other lanes
                // idle for the whole row); past the list's end, here
                const uint32_t slot = atomicAdd(&s_nrl, 1u);
                if (slot < kRecheckCap) {
                    s_rl[slot] = (uint16_t)((j << 7) | i);
                    continue;
                }
                dji = fp32_pair(j, i);
                if (a.rechecks) atomicAdd(a.rechecks, 1ull);
            }
        }
        if (a.alpha2 * dji < s_d[i]) atomicOr(&s_occ[j][i >> 5], 1u << (i & 31));
    }
    __syncthreads();
    if (TC) {
        const uint32_t nrl = min(s_nrl, kRecheckCap);
        for (uint32_t t = tid; t < nrl; t += kPruneThreads) {
            const uint32_t j = s_rl[t] >> 7, i = s_rl[t] & 127u;
            if (a.alpha2 * fp32_pair(j, i) < s_d[i]) atomicOr(&s_occ[j][i >> 5], 1u << (i & 31));
        }
        if (a.rechecks && tid == 0 && nrl) atomicAdd(a.rechecks, (unsigned long long)nrl);
        __syncthreads();
    }

    // 5b. the greedy pass over the bit rows, in one warp: candidates in
    // distance order; an open one is kept (within the caps) and prunes what
    // its row marks.
    const uint32_t cap = a.out_cap ? min(a.out_cap, a.deg) : a.deg;
    // far_budget slots are held for long links: a candidate farther than 4x
    // the nearest one's squared distance; near ones stop at cap - far_budget
    const uint32_t near_cap = a.far_budget < cap ? cap - a.far_budget : cap;
    const float far_d = 4.0f * s_d[0];
    if (tid < 32) {
        uint32_t pruned[kOccW];
#pragma unroll
        for (uint32_t w = 0; w < kOccW; ++w) pruned[w] = 0;
        uint32_t kept_n = 0, kept_near = 0;
        for (uint32_t j = 0; j < P; ++j) {
            if ((pruned[j >> 5] >> (j & 31)) & 1u) continue;
            if (kept_n >= cap) break;
            const bool is_far = a.far_budget != 0 && s_d[j] > far_d;
            if (!is_far && kept_near >= near_cap) continue;
            ++kept_n;
            if (!is_far) ++kept_near;
            if (tid == 0) s_keep[j] = 1;
#pragma unroll
            for (uint32_t w = 0; w < kOccW; ++w) pruned[w] |= s_occ[j][w];
        }
    }
    __syncthreads();
    // 5c. the output lists, compacted by warp 0 with ballots: kept ones in
    // distance order, then (fill) the others, then (rest_fill) the caller's
    // earlier list without duplicates, all cut at cap
    if (tid < 32) {
        constexpr uint32_t kOutMax = 128;  // degree_bound's largest value
        __shared__ uint32_t s_out[kOutMax];
        const uint32_t lt = (1u << tid) - 1u;
        uint32_t w = 0;
        for (uint32_t j0 = 0; j0 < P && w < cap; j0 += 32) {
            const uint32_t j = j0 + tid;
            const bool take = j < P && s_keep[j];
            const uint32_t m = __ballot_sync(~0u, take);
            const uint32_t pos = w + __popc(m & lt);
            if (take && pos < cap) s_out[pos] = s_ids[j] >> 1;
            w = min(w + __popc(m), cap);
        }
        const uint32_t kept = w;
        if (a.fill)
            for (uint32_t j0 = 0; j0 < P && w < cap; j0 += 32) {
                const uint32_t j = j0 + tid;
                const bool take = j < P && !s_keep[j];
                const uint32_t m = __ballot_sync(~0u, take);
                const uint32_t pos = w + __popc(m & lt);
                if (take && pos < cap) s_out[pos] = s_ids[j] >> 1;
                w = min(w + __popc(m), cap);
            }
        __syncwarp();
        if (a.rest_fill) {  // caller's earlier pruned list
            const uint32_t* rr = a.rest_fill + node * a.rest_stride;
            const uint32_t rc = min(a.rest_fill_cnt[node], a.rest_stride);
            for (uint32_t j0 = 0; j0 < rc && w < cap; j0 += 32) {
                const uint32_t j = j0 + tid;
                const bool in = j < rc;
                const uint32_t v = in ? rr[j] : 0xFFFFFFFFu;
                bool dup = !in || v == (uint32_t)node;
                for (uint32_t t = 0; t < w && !dup; ++t) dup = s_out[t] == v;
                // a lower lane with the same id: that one is taken or is itself
                // a duplicate, so this one is a duplicate either way
                if (__match_any_sync(~0u, v) & lt) dup = true;
                const uint32_t m = __ballot_sync(~0u, !dup);
                const uint32_t pos = w + __popc(m & lt);
                if (!dup && pos < cap) s_out[pos] = v;
                w = min(w + __popc(m), cap);
                __syncwarp();
            }
        }
        uint32_t* out = a.out + node * a.deg;
        for (uint32_t t = tid; t < w; t += 32) out[t] = s_out[t];
        if (a.rest) {
            uint32_t* rr = a.rest + node * a.rest_stride;
            uint32_t rw = 0;
            for (uint32_t j0 = 0; j0 < P && rw < a.rest_stride; j0 += 32) {
                const uint32_t j = j0 + tid;
                const bool take = j < P && !s_keep[j];
                const uint32_t m = __ballot_sync(~0u, take);
                const uint32_t pos = rw + __popc(m & lt);
                if (take && pos < a.rest_stride) rr[pos] = s_ids[j] >> 1;
                rw = min(rw + __popc(m), a.rest_stride);
            }
            if (tid == 0) a.rest_cnt[node] = rw;
        }
        if (tid == 0) {
            a.out_cnt[node] = w;
            if (a.kept_cnt) a.kept_cnt[node] = kept;
        }
    }
}

size_t prune_smem_bytes(int tc) {
    const size_t tile = tc ? (size_t)128 * kTileD : (size_t)(kPruneMax + 1) * (kTileD + 1);
    return sizeof(float) * (tile + (size_t)kPruneMax * kPruneMax);
}

// Reverse lists as CSR, deterministic: pair (target, source) for every kept
// edge at a fixed position, a stable radix sort by target, then each target's
// segment [start, end) of sources in ascending source order.
__global__ void reverse_pairs_kernel(const uint32_t* __restrict__ nb,
                                     const uint32_t* __restrict__ cnt, uint64_t n, uint32_t deg,
                                     uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * deg) return;
    const uint64_t node = e / deg;
    const uint32_t j = (uint32_t)(e % deg);
    const bool ok = j < min(cnt[node], deg);
    keys[e] = ok ? nb[e] : 0xFFFFFFFFu;
    vals[e] = (uint32_t)node;
}

__global__ void segment_kernel(const uint32_t* __restrict__ keys, uint64_t total, uint64_t n,
                               uint32_t* __restrict__ start, uint32_t* __restrict__ end) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint32_t k = keys[i];
    if (k >= n) return;
    if (i == 0 || keys[i - 1] != k) start[k] = (uint32_t)i;
    if (i + 1 == total || keys[i + 1] != k) end[k] = (uint32_t)(i + 1);
}

cudaError_t launch_prune(const PruneArgs& a, uint64_t nodes, cudaStream_t st) {
    const size_t smem = prune_smem_bytes(a.pair_tc);
    auto k = a.pair_tc ? prune_kernel<1> : prune_kernel<0>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<(unsigned)nodes, kPruneThreads, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sq8_encode(const float* x, uint64_t n, uint32_t dim, float* params,
                              uint8_t* codes, float* work, cudaStream_t st) {
    const uint32_t nb = 1024;
    const uint64_t rpb = (n + nb - 1) / nb;
    minmax_partial_kernel<<<nb, 128, 0, st>>>(x, n, dim, rpb, work, work + (size_t)nb * dim);
    minmax_final_kernel<<<(dim + 127) / 128, 128, 0, st>>>(work, work + (size_t)nb * dim, nb, dim,
                                                           params);
    sq8_encode_kernel<<<4096, 256, 0, st>>>(x, n * dim, dim, params, codes);
    return cudaGetLastError();
}

size_t sq8_work_floats(uint32_t dim) { return 2 * 1024 * (size_t)dim; }

cudaError_t launch_entry(const float* x, uint64_t n, uint32_t dim, double* work, float* centroid,
                         unsigned long long* best, cudaStream_t st) {
    const uint32_t nb = 1024;
    const uint64_t rpb = (n + nb - 1) / nb;
    centroid_partial_kernel<<<nb, 128, 0, st>>>(x, n, dim, rpb, work);
    centroid_final_kernel<<<(dim + 127) / 128, 128, 0, st>>>(work, nb, dim, n, centroid);
    cudaMemsetAsync(best, 0xFF, sizeof(unsigned long long), st);
    nearest_kernel<<<1024, 256, 0, st>>>(x, n, dim, centroid, best);
    return cudaGetLastError();
}

size_t entry_work_doubles(uint32_t dim) { return 1024 * (size_t)dim; }

cudaError_t launch_random_fill(uint32_t* out, const uint32_t* from, uint64_t n, uint32_t deg,
                               uint64_t seed, cudaStream_t st) {
    const uint64_t threads = n * 32;
    random_fill_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(out, from, n, deg, seed);
    return cudaGetLastError();
}

size_t reverse_temp_bytes(uint64_t n, uint32_t deg) {
    size_t t = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)(n * deg));
    return t;
}

cudaError_t launch_reverse(const uint32_t* nb, const uint32_t* cnt, uint64_t n, uint32_t deg,
                           ReverseWork& w, cudaStream_t st) {
    const uint64_t total = n * deg;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    reverse_pairs_kernel<<<blocks, 256, 0, st>>>(nb, cnt, n, deg, w.keys_in, w.vals_in);
    size_t tb = w.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(w.temp, tb, w.keys_in, w.keys_out, w.vals_in,
                                                    w.vals_out, (int)total, 0, 32, st);
    if (e != cudaSuccess) return e;
    cudaMemsetAsync(w.start, 0, n * sizeof(uint32_t), st);
    cudaMemsetAsync(w.end, 0, n * sizeof(uint32_t), st);
    segment_kernel<<<blocks, 256, 0, st>>>(w.keys_out, total, n, w.start, w.end);
    return cudaGetLastError();
}

}  // namespace lqg
