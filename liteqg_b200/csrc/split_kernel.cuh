// Split search kernel: the reference's search loop (QuantizedGraph::
// search_qg_with_heap, symqglib/qg/qg.hpp:298-344), exact for every query,
// ties included, with the result pool's heap work moved to a later pass.
//
// One warp per query, persistent over the work queue. The search pool `sp`
// is the reference's std::priority_queue emulated step for step in shared
// memory (heap_ops.cuh), so every pop is the reference's pop, equal
// distances included. Of the result pool `rp` the search needs only its size,
// min(accepted, ef), and lowerBound = rp.top().distance, which is the ef-th
// smallest accepted distance (each trim removes a largest element, so rp's
// multiset of distances is the ef smallest accepted ones; while rp is not full
// it is the largest accepted one). The warp keeps the accepted nodes at or
// below the bound sorted in registers (E entries per lane) for that, and
// appends every accepted node, in order, to the query's result log in HBM
// (id, distance, bound after). When the output does not depend on how equal
// distances sit in rp (below), the warp writes it from the sorted array;
// otherwise rp_replay_kernel (replay_launch.cu) replays the log on a result
// heap laid out exactly as libstdc++ leaves it, checks every acceptance
// against the reference's test on that heap and the logged bound against
// rp.top(), and writes the output (qg.hpp:340-343).
//
// Visited set: the direct-mapped cache of evaluated ids in shared memory. It
// may forget an id, never invents one. A forgotten node that is evaluated
// again has its old distance; if it passes the acceptance test now, it was
// accepted before and is still in the register array (at or below the bound)
// with the same id and distance, and it is dropped there.
//
// A query whose search pool, sorted array or log outgrows its capacity goes to
// the exact global-memory kernel through the spill list.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>

#include "heap_ops.cuh"
#include "lqg_internal.h"
#include "lqg_kernels.cuh"
#include "sq8_batch.cuh"

namespace lqg {

template <int E>
__device__ __forceinline__ float spool_at(const float (&pd)[E], uint32_t pos) {
    const uint32_t l = pos / E, s = pos % E;
    float v = pd[0];
#pragma unroll
    for (int t = 1; t < E; ++t)
        if (s == (uint32_t)t) v = pd[t];
    return __shfl_sync(kFull, v, l);
}

__host__ __device__ inline size_t split_warp_bytes(uint32_t dim, uint32_t vbits, uint32_t scap) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 4 * dpad + 4 * ((size_t)1 << vbits) + kCandBytes + 8 * (size_t)scap;
}

// After a search, a warp's visited cache, candidates and search heap can
// hold a result heap of rcap slots.
__host__ __device__ inline bool split_replays_in_place(uint32_t vbits, uint32_t scap, uint32_t rcap) {
    return 4 * ((size_t)1 << vbits) + kCandBytes + 8 * (size_t)scap >= 8 * (size_t)rcap;
}

// At most 5 warps per block and 96 registers per thread, so 20 warps (queries)
// fit on an SM.
template <int E, int G, int DEGW>
__global__ void __launch_bounds__(160, 4) split_search_kernel(SearchArgs a, ReplayArgs ra) {
    using namespace heapops;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t dim = a.dim;
    const uint32_t dpad = (dim + 15u) & ~15u;
    float* pmin = reinterpret_cast<float*>(smem);
    float* pscale = pmin + dpad;
    const uint32_t vbits = a.vbits;
    const uint32_t vsize = 1u << vbits;
    unsigned char* wb = smem + 8u * dpad + (size_t)warp * split_warp_bytes(dim, vbits, ra.scap);
    float* qs = reinterpret_cast<float*>(wb);
    uint32_t* vis = reinterpret_cast<uint32_t*>(wb + 4u * dpad);
    uint32_t* cid = vis + vsize;
    float* cd = reinterpret_cast<float*>(cid + kMaxDeg);
    uint2* sps = reinterpret_cast<uint2*>(cd + kMaxDeg);
    const size_t gw = (size_t)blockIdx.x * (blockDim.x >> 5) + warp;
    const HeapView sp{sps, ra.sp_global + gw * ra.gcap, ra.scap};
    const uint32_t sp_max = ra.scap + ra.gcap;

    for (uint32_t i = threadIdx.x; i < dpad; i += blockDim.x) {
        pmin[i] = i < dim ? a.params[2 * i] : 0.f;
        pscale[i] = i < dim ? a.params[2 * i + 1] : 0.f;
    }
    __syncthreads();

    const int g = lane / G, r = lane % G;
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
        ef = min(max(ef, 1u), ra.efcap);  // efcap <= 32 E - 32
        const float* q = a.queries + (size_t)qi * dim;
        uint4* rlog = ra.rlog + (size_t)qi * ra.rlog_cap;
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
        // qg.hpp:305-311: the entry point seeds both pools and is visited
        const uint32_t ep = a.entry;
        if (lane == 0) cid[0] = ep;
        __syncwarp();
        eval_batch<G, G>(a, cid, cd, 0, 1, qs, pmin, pscale, g, r);
        __syncwarp();
        const float d0 = cd[0];
        bool fail = !(d0 < INF);
        uint32_t acc_n = 1;  // accepted so far (rp.size() = min(acc_n, ef))
        float lower = d0;
        uint32_t sn = 1;
        if (lane == 0) {
            sp.set(0, make_uint2(ep, __float_as_uint(-d0)));
            pd[0] = d0;
            pi[0] = ep;
            vis[hash_id(ep, vbits)] = ep;
            rlog[0] = make_uint4(ep, __float_as_uint(d0), __float_as_uint(d0), 0u);
        }
        __syncwarp();
        uint32_t pops = 0, calcs = 1;

        while (!fail) {
            // qg.hpp:313-318
            if (sn == 0) break;
            const uint2 top = sp.get(0);
            if (-__uint_as_float(top.y) > lower) break;
            warp_pop(sp, sn, lane);
            const uint32_t u = top.x;
            ++pops;

            // qg.hpp:320-324: unvisited neighbours in list order
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

            // qg.hpp:325-328
            for (uint32_t b = 0; b < ncand; b += 32)
                eval_batch<G, G>(a, cid, cd, b, ncand, qs, pmin, pscale, g, r);
            calcs += ncand;
            __syncwarp();

            // qg.hpp:329-335, in list order
            const bool full0 = acc_n >= ef;
            const float lower0 = lower;
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t c0 = w * 32;
                if (c0 >= ncand) break;
                const uint32_t c = c0 + lane;
                const float dc = c < ncand ? cd[c] : 0.f;
                if (__any_sync(kFull, c < ncand && !(dc < INF))) {
                    fail = true;
                    break;
                }
                const bool pass = c < ncand && (!full0 || lower0 > dc);
                unsigned pm = __ballot_sync(kFull, pass);
                while (pm) {
                    const int src = __ffs(pm) - 1;
                    pm &= pm - 1;
                    const float y = __shfl_sync(kFull, dc, src);
                    if (!(acc_n < ef || lower > y)) continue;
                    const uint32_t id = cid[c0 + src];
                    // a node the visited cache forgot: still pooled, same distance
                    bool dup = false;
#pragma unroll
                    for (int t = 0; t < E; ++t) dup |= pd[t] == y && pi[t] == id;
                    if (__any_sync(kFull, dup)) continue;
                    // room in the sorted array (ties at the bound can exceed ef),
                    // the log and the search pool
                    if (__shfl_sync(kFull, pd[E - 1], 31) < INF || acc_n >= ra.rlog_cap ||
                        sn + 1 > sp_max) {
                        fail = true;
                        break;
                    }
                    warp_push(sp, sn, make_uint2(id, __float_as_uint(-y)), lane);
                    uint32_t cl = 0;
#pragma unroll
                    for (int t = 0; t < E; ++t) cl += pd[t] <= y ? 1u : 0u;
                    const uint32_t p = __reduce_add_sync(kFull, cl);
                    const float pdp = __shfl_up_sync(kFull, pd[E - 1], 1);
                    const uint32_t pip = __shfl_up_sync(kFull, pi[E - 1], 1);
#pragma unroll
                    for (int t = E - 1; t >= 0; --t) {
                        const uint32_t pos = (uint32_t)lane * E + t;
                        float nd = t > 0 ? pd[t > 0 ? t - 1 : 0] : pdp;
                        uint32_t ni = t > 0 ? pi[t > 0 ? t - 1 : 0] : pip;
                        if (pos == p) {
                            nd = y;
                            ni = id;
                        }
                        if (pos >= p) {
                            pd[t] = nd;
                            pi[t] = ni;
                        }
                    }
                    lower = spool_at<E>(pd, min(acc_n + 1, ef) - 1);
                    if (acc_n + 1 > ef) {
                        // beyond the ef-th entry only ties with the bound stay
#pragma unroll
                        for (int t = 0; t < E; ++t) {
                            const uint32_t pos = (uint32_t)lane * E + t;
                            if (pos >= ef && pd[t] > lower) {
                                pd[t] = INF;
                                pi[t] = kNoId;
                            }
                        }
                    }
                    if (lane == 0)
                        rlog[acc_n] = make_uint4(id, __float_as_uint(y), __float_as_uint(lower), 0u);
                    ++acc_n;
                }
                if (fail) break;
            }
        }

        // Output (qg.hpp:340-343). rp pops come out in descending distance;
        // only equal distances make the heap layout decide. So when the
        // sorted array holds exactly rp (no ties beyond the ef-th entry) and
        // the popped entries (the worst k and the one after them, or the
        // whole pool when it is returned) have distinct distances, the output
        // is read off the array; otherwise the result replay pass computes it.
        const uint32_t P = min(acc_n, ef);
        bool direct = false;
        if (!fail && !ra.replay_all) {
            const uint32_t k = min(a.kq ? a.kq[qi] : a.k0, a.kstride);
            const uint32_t kk = min(k, P);
            const uint32_t lo = a.pool_ids ? 0u : (P > kk ? P - kk - 1 : 0u);
            const float nx0 = __shfl_down_sync(kFull, pd[0], 1);
            uint32_t vc = 0;
            bool tie = false;
#pragma unroll
            for (int t = 0; t < E; ++t) {
                const uint32_t pos = (uint32_t)lane * E + t;
                vc += pd[t] < INF ? 1u : 0u;
                const float nxt = t + 1 < E ? pd[t + 1 < E ? t + 1 : 0] : nx0;
                if (pos >= lo && pos + 1 < P && pd[t] == nxt) tie = true;
            }
            direct = __reduce_add_sync(kFull, vc) == P && !__any_sync(kFull, tie);
            if (direct) {
                uint32_t* out = a.ids + (size_t)qi * a.kstride;
                for (uint32_t x = lane; x < k - kk; x += 32) out[x] = kNoId;
#pragma unroll
                for (int t = 0; t < E; ++t) {
                    const uint32_t pos = (uint32_t)lane * E + t;
                    if (pos < P && pos + kk >= P) out[pos + k - P] = pi[t];
                    if (a.pool_ids && pos < P && pos < a.pstride) {
                        a.pool_ids[(size_t)qi * a.pstride + pos] = pi[t];
                        a.pool_d[(size_t)qi * a.pstride + pos] = pd[t];
                    }
                }
                if (a.pool_ids)
                    for (uint32_t x = P + lane; x < a.pstride; x += 32) {
                        a.pool_ids[(size_t)qi * a.pstride + x] = kNoId;
                        a.pool_d[(size_t)qi * a.pstride + x] = INF;
                    }
            }
        }
        // an output the heap layout decides: replay rp here, in this warp's
        // shared memory (its visited cache, candidates and search heap are
        // free now), else in the result replay pass
        if (!fail && !direct && !ra.replay_all && split_replays_in_place(vbits, ra.scap, ra.rcap)) {
            __syncwarp();
            const HeapView rph{reinterpret_cast<uint2*>(vis), nullptr, ra.rcap};
            fail = !replay_result(a, ra, qi, acc_n, rph, lane);
            direct = !fail;
        }
        if (lane == 0) {
            ra.rlen[qi] = fail ? kNoId : (direct ? kRlenDone : acc_n);
            if (fail) {
                const uint32_t i = atomicAdd(ra.nspill, 1u);
                ra.spill[i] = (int32_t)qi;
            }
            if (a.stats) {
                *reinterpret_cast<uint4*>(a.stats + 4 * (size_t)qi) =
                    make_uint4(pops, calcs, 0u, P);
            }
        }
        __syncwarp();
    }
}

template <int E, int G, int DEGW>
static cudaError_t split_run(const SearchArgs& a, const ReplayArgs& ra, int warps, int blocks,
                            cudaStream_t st, int* occ) {
    const size_t dpad = (a.dim + 15u) & ~15u;
    const size_t smem = 8 * dpad + (size_t)warps * split_warp_bytes(a.dim, a.vbits, ra.scap);
    auto k = split_search_kernel<E, G, DEGW>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, warps * 32, smem);
    k<<<blocks, warps * 32, smem, st>>>(a, ra);
    return cudaGetLastError();
}

// All instances for one sorted-array size E: lanes per candidate x degree words.
template <int E>
cudaError_t split_dispatch(const SearchArgs& a, const ReplayArgs& ra, int G, int degw, int warps,
                           int blocks, cudaStream_t st, int* occ) {
#define LQG_SCASE(GG, DW) \
    if (G == GG && degw == DW) return split_run<E, GG, DW>(a, ra, warps, blocks, st, occ);
#define LQG_SCASES(GG) LQG_SCASE(GG, 1) LQG_SCASE(GG, 2) LQG_SCASE(GG, 3) LQG_SCASE(GG, 4)
    LQG_SCASES(2)
    LQG_SCASES(4)
    LQG_SCASES(8)
#undef LQG_SCASES
#undef LQG_SCASE
    return cudaErrorInvalidValue;
}

}  // namespace lqg
