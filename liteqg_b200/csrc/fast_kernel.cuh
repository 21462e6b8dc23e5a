// Fast search kernel template (instantiated in fast_e*.cu).
// The two search kernels of the B200 query path, and their launchers.
//
// Reference: QuantizedGraph::search_qg_with_heap, symqglib/qg/qg.hpp:298-344
// (best-first search over a search pool `sp` and an ef-bounded result pool
// `rp`, both std::priority_queue, with an exact visited set).
//
// fast_search_kernel — one warp per query, persistent over a work queue.
//   When no two distances that meet in the pools are equal, the reference's
//   loop is exactly: "while the ef-pool holds an unexpanded node, expand the
//   nearest one; every unvisited neighbour gets a distance; the pool becomes
//   the ef smallest of (pool + neighbours)". Items the reference pushes on
//   sp but later trims from rp are then strictly above every later bound and
//   never pop. The kernel therefore keeps only the ef-pool, sorted, in
//   registers (E entries per lane), with the "expanded" bit in the id.
//   The visited set is a direct-mapped cache of evaluated ids in shared
//   memory: it may forget an id but never reports an unvisited one, and a
//   forgotten id that is evaluated again has the same distance, so it either
//   fails the bound or meets its own pool entry (same id, same distance) and
//   is dropped. Candidates are merged in ascending distance; any equality
//   between a candidate and the pool, or between two candidates, with
//   different ids (or a non-finite distance) hands the query to the exact
//   kernel, since only there does the reference's heap layout decide.
//
// exact_search_kernel — one warp per query from a list. Emulates the
//   reference literally: sp/rp as GCC libstdc++ binary heaps in global
//   memory (push = sift-up; pop = hole to leaf along the larger child, then
//   sift-up), an exact visited hash set, neighbours accepted in list order.
//   Lanes share the distance work; lane 0 runs the heaps.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>

#include "lqg_internal.h"
#include "lqg_kernels.cuh"
#include "sq8_batch.cuh"

namespace lqg {

// Code words in flight per lane in the fast kernel's distance batches: the
// 512-entry pool (E = 16) holds 32 registers per lane, so it gets the short
// window.
template <int E>
constexpr int kFastLoadWords = E >= 16 ? 8 : 16;

template <int E>
__device__ __forceinline__ float pool_at(const float (&pd)[E], uint32_t lane_of, uint32_t slot_of) {
    float v = pd[0];
#pragma unroll
    for (int t = 1; t < E; ++t)
        if (slot_of == (uint32_t)t) v = pd[t];
    return __shfl_sync(kFull, v, lane_of);
}

template <int E, int G, int DEGW>
__global__ void __launch_bounds__(512) fast_search_kernel(SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t dim = a.dim;
    const uint32_t dpad = (dim + 15u) & ~15u;
    float* pmin = reinterpret_cast<float*>(smem);
    float* pscale = pmin + dpad;
    const uint32_t vbits = a.vbits;
    const uint32_t vsize = 1u << vbits;
    unsigned char* wb = smem + 8u * dpad + (size_t)warp * (4u * dpad + 4u * vsize + kCandBytes);
    float* qs = reinterpret_cast<float*>(wb);
    uint32_t* vis = reinterpret_cast<uint32_t*>(wb + 4u * dpad);
    uint32_t* cid = vis + vsize;
    float* cd = reinterpret_cast<float*>(cid + kMaxDeg);

    for (uint32_t i = threadIdx.x; i < dpad; i += blockDim.x) {
        pmin[i] = i < dim ? a.params[2 * i] : 0.f;
        pscale[i] = i < dim ? a.params[2 * i + 1] : 0.f;
    }
    __syncthreads();

    const int g = lane / G, r = lane % G;
    constexpr int CPP = 32 / G;
    const uint32_t lt = lanemask_lt();
    const int64_t mlist = a.nlist ? (int64_t)*a.nlist : a.m;
    const float INF = CUDART_INF_F;

    for (;;) {
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(a.qhead, 1u);
        slot = __shfl_sync(kFull, slot, 0);
        if ((int64_t)slot >= mlist) break;
        const int64_t qi = a.qlist ? (int64_t)a.qlist[slot] : (int64_t)slot;
        uint32_t ef = query_ef(a, qi);
        ef = min(max(ef, 1u), 32u * E);
        const uint32_t k = min(a.kq ? a.kq[qi] : a.k0, a.kstride);
        const float* q = a.queries + (size_t)qi * dim;
        for (uint32_t i = lane; i < dpad; i += 32) qs[i] = i < dim ? q[i] : 0.f;
        for (uint32_t i = lane; i < vsize; i += 32) vis[i] = kNoId;
        __syncwarp();

        float pd[E];
        uint32_t pi[E];
#pragma unroll
        for (int t = 0; t < E; ++t) {
            pd[t] = INF;
            pi[t] = kNoId;
        }

        // qg.hpp:305-311: the entry point seeds both pools and is visited.
        const uint32_t ep = a.entry;
        float d0 = sq8_l2_group<G>(a.codes + (size_t)ep * a.cstride, g == 0, qs, pmin,
                                   pscale, dim, r);
        d0 = __shfl_sync(kFull, d0, 0);
        bool tie = !(d0 < INF) && !a.ties_ok;
        if (lane == 0) {
            pd[0] = d0;
            pi[0] = ep;
            vis[hash_id(ep, vbits)] = ep;
        }
        __syncwarp();
        uint32_t pops = 0, calcs = 1;
        const uint32_t tl = (ef - 1) / E, ts = (ef - 1) % E;  // position ef-1
        const bool trim = ef < 32u * E;
        const uint32_t cl = ef / E, cs = ef % E;  // position ef

        while (!tie) {
            // qg.hpp:313-318: pop the nearest unexpanded pool entry.
            int tf = E;
#pragma unroll
            for (int t = E - 1; t >= 0; --t)
                if (!(pi[t] & kExpanded)) tf = t;
            const unsigned hb = __ballot_sync(kFull, tf < E);
            if (!hb) break;
            const int owner = __ffs(hb) - 1;
            uint32_t u = 0;
            if (lane == owner) {
#pragma unroll
                for (int t = 0; t < E; ++t)
                    if (t == tf) {
                        u = pi[t];
                        pi[t] |= kExpanded;
                    }
            }
            u = __shfl_sync(kFull, u, owner);
            if (a.path && pops < a.path_stride && lane == 0)
                a.path[(size_t)qi * a.path_stride + pops] = u;
            ++pops;

            // qg.hpp:320-324: neighbours in list order, unvisited ones kept.
            uint32_t ncand = 0;
            const uint32_t* nb = a.nbrs + (size_t)u * a.deg;
            uint32_t v[DEGW];
#pragma unroll
            for (int w = 0; w < DEGW; ++w) v[w] = __ldg(nb + w * 32 + lane);
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t h = hash_id(v[w], vbits);
                const bool seen = vis[h] == v[w];
                const unsigned mm = __match_any_sync(kFull, v[w]);
                const bool keep = !seen && (mm & lt) == 0;
                __syncwarp();
                if (keep) vis[h] = v[w];
                const unsigned kb = __ballot_sync(kFull, keep);
                if (keep) cid[ncand + __popc(kb & lt)] = v[w];
                ncand += __popc(kb);
                __syncwarp();
            }

            // qg.hpp:325-328: SQ8 decode + L2 of every kept neighbour. Rows
            // below 256 bytes with up to 4 lanes per candidate: the packed-pair
            // batch routine (32 candidates per call, code loads of every pass
            // issued before the arithmetic; the same operations in the same
            // order). Longer rows, or wider groups: one candidate per group at
            // a time with 8 chunks of the row in flight (the batch routine's
            // short load window would take a dependent round per two chunks).
            bool packed = false;
            if constexpr (G <= 4) packed = dim < kBatchWideDim;
            if (packed) {
                if constexpr (G <= 4)
                    for (uint32_t b = 0; b < ncand; b += 32)
                        eval_batch<G, G, kFastLoadWords<E>, 1>(a, cid, cd, b, ncand, qs, pmin,
                                                               pscale, g, r);
            } else {
                for (uint32_t base = 0; base < ncand; base += CPP) {
                    const uint32_t c = base + g;
                    const bool valid = c < ncand;
                    const uint32_t id = valid ? cid[c] : 0u;
                    const float d = sq8_l2_group<G>(a.codes + (size_t)id * a.cstride, valid, qs,
                                                    pmin, pscale, dim, r);
                    if (valid && r == 0) cd[c] = d;
                }
            }
            calcs += ncand;
            __syncwarp();

            // qg.hpp:329-335: pool <- ef smallest of (pool + candidates).
            float T = pool_at<E>(pd, tl, ts);
            uint32_t key[DEGW], cv[DEGW];
            bool bad = false;
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t c = w * 32 + lane;
                const bool valid = c < ncand;
                const float dc = valid ? cd[c] : INF;
                cv[w] = valid ? cid[c] : 0u;
                bad |= valid && !(dc < INF);
                key[w] = (valid && dc < T) ? __float_as_uint(dc) : 0xFFFFFFFFu;
            }
            if (__any_sync(kFull, bad) && !a.ties_ok) {
                tie = true;
                break;
            }
            for (;;) {
                uint32_t lk = key[0];
#pragma unroll
                for (int w = 1; w < DEGW; ++w) lk = min(lk, key[w]);
                const uint32_t mn = __reduce_min_sync(kFull, lk);
                if (mn == 0xFFFFFFFFu) break;
                int src_w = DEGW - 1;
#pragma unroll
                for (int w = DEGW - 1; w >= 0; --w)
                    if (key[w] == mn) src_w = w;
                const unsigned hold = __ballot_sync(kFull, lk == mn);
                const int src = __ffs(hold) - 1;
                uint32_t mine = cv[0];
#pragma unroll
                for (int w = 1; w < DEGW; ++w)
                    if (src_w == w) mine = cv[w];
                const uint32_t cidv = __shfl_sync(kFull, mine, src);
                // holders of the same id are one node: drop them; a holder
                // with another id is a tie (left in place for ties_ok)
                bool other = false;
#pragma unroll
                for (int w = 0; w < DEGW; ++w)
                    if (key[w] == mn) {
                        if (cv[w] != cidv) other = true;
                        else key[w] = 0xFFFFFFFFu;
                    }
                if (__any_sync(kFull, other) && !a.ties_ok) {
                    tie = true;
                    break;
                }
                const float dmin = __uint_as_float(mn);
                bool dup = false, teq = false;
#pragma unroll
                for (int t = 0; t < E; ++t)
                    if (pd[t] == dmin) {
                        if ((pi[t] & ~kExpanded) == cidv) dup = true;
                        else teq = true;
                    }
                if (__any_sync(kFull, dup)) continue;  // the same node again: already pooled
                if (__any_sync(kFull, teq) && !a.ties_ok) {
                    tie = true;
                    break;
                }
                if (!(dmin < T)) break;
                uint32_t cnt = 0;
#pragma unroll
                for (int t = 0; t < E; ++t) cnt += pd[t] < dmin ? 1u : 0u;
                const uint32_t p = __reduce_add_sync(kFull, cnt);
                const float pdp = __shfl_up_sync(kFull, pd[E - 1], 1);
                const uint32_t pip = __shfl_up_sync(kFull, pi[E - 1], 1);
#pragma unroll
                for (int t = E - 1; t >= 0; --t) {
                    const uint32_t pos = (uint32_t)lane * E + t;
                    float nd = t > 0 ? pd[t > 0 ? t - 1 : 0] : pdp;
                    uint32_t ni = t > 0 ? pi[t > 0 ? t - 1 : 0] : pip;
                    if (pos == p) {
                        nd = dmin;
                        ni = cidv;
                    }
                    if (pos >= p) {
                        pd[t] = nd;
                        pi[t] = ni;
                    }
                }
                if (trim && (uint32_t)lane == cl) {
#pragma unroll
                    for (int t = 0; t < E; ++t)
                        if ((uint32_t)t == cs) {
                            pd[t] = INF;
                            pi[t] = kNoId;
                        }
                }
                T = pool_at<E>(pd, tl, ts);
            }
        }

        if (tie) {
            if (lane == 0) {
                const uint32_t i = atomicAdd(a.nflagged, 1u);
                a.flagged[i] = (int32_t)qi;
            }
            continue;
        }

        // qg.hpp:340-343: results[k-1-j] = j-th largest of the pool.
        uint32_t cntv = 0;
#pragma unroll
        for (int t = 0; t < E; ++t) cntv += pd[t] < INF ? 1u : 0u;
        const uint32_t P = __reduce_add_sync(kFull, cntv);
        const uint32_t kk = min(k, P);
        uint32_t* out = a.ids + (size_t)qi * a.kstride;
        for (uint32_t j = lane; j < k - kk; j += 32) out[j] = kNoId;
#pragma unroll
        for (int t = 0; t < E; ++t) {
            const uint32_t pos = (uint32_t)lane * E + t;
            if (pos < P && pos + kk >= P) out[pos + k - P] = pi[t] & ~kExpanded;
        }
        if (a.pool_ids) {
            uint32_t* po = a.pool_ids + (size_t)qi * a.pstride;
            float* pdo = a.pool_d + (size_t)qi * a.pstride;
#pragma unroll
            for (int t = 0; t < E; ++t) {
                const uint32_t pos = (uint32_t)lane * E + t;
                if (pos < P && pos < a.pstride) {
                    po[pos] = pi[t] & ~kExpanded;
                    pdo[pos] = pd[t];
                }
            }
            for (uint32_t j = P + lane; j < a.pstride; j += 32) {
                po[j] = kNoId;
                pdo[j] = INF;
            }
        }
        if (a.path)
            for (uint32_t j = pops + lane; j < a.path_stride; j += 32)
                a.path[(size_t)qi * a.path_stride + j] = kNoId;
        if (a.stats && lane == 0) {
            uint4 st = make_uint4(pops, calcs, 0u, P);
            *reinterpret_cast<uint4*>(a.stats + 4 * (size_t)qi) = st;
        }
    }
}

template <int E, int G, int DEGW>
static cudaError_t run_fast(const SearchArgs& a, int warps, int blocks, size_t smem,
                            cudaStream_t st) {
    auto k = fast_search_kernel<E, G, DEGW>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k<<<blocks, warps * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int E, int G, int DEGW>
static int occ_of(int warps, size_t smem) {
    auto k = fast_search_kernel<E, G, DEGW>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, warps * 32, smem) != cudaSuccess)
        return 0;
    return nb;
}

// All instances for one pool size E: lanes per candidate G x degree words.
template <int E>
cudaError_t fast_dispatch(const SearchArgs& a, int G, int degw, int warps, int blocks,
                          size_t smem, cudaStream_t st, int* occ) {
#define LQG_CASE(GG, DW)                                              \
    if (G == GG && degw == DW) {                                      \
        if (occ) {                                                    \
            *occ = occ_of<E, GG, DW>(warps, smem);                    \
            return cudaSuccess;                                       \
        }                                                             \
        return run_fast<E, GG, DW>(a, warps, blocks, smem, st);       \
    }
#define LQG_CASES(GG) LQG_CASE(GG, 1) LQG_CASE(GG, 2) LQG_CASE(GG, 3) LQG_CASE(GG, 4)
    LQG_CASES(1)
    LQG_CASES(2)
    LQG_CASES(4)
    LQG_CASES(8)
    LQG_CASES(16)
#undef LQG_CASES
#undef LQG_CASE
    return cudaErrorInvalidValue;
}

}  // namespace lqg
