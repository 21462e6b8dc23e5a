// Batched-acceptance search kernel: the reference's search loop
// (QuantizedGraph::search_qg_with_heap, symqglib/qg/qg.hpp:298-344), exact
// for every query, ties included.
//
// One warp per query, persistent over the work queue, as the split kernel:
// the search pool `sp` is the reference's std::priority_queue emulated step
// for step (heap_ops.cuh), and of the result pool `rp` the search keeps only
// what it reads, lowerBound = rp.top().distance, the ef-th smallest accepted
// distance (the largest one while fewer than ef are accepted). The accepted
// nodes at or below the bound are kept sorted in shared memory (the sorted
// pool), and every accepted node is appended, in order, to the query's result
// log in HBM (id, distance, bound after it).
//
// What differs is how one expansion's candidates are decided. The reference
// takes them one by one in list order (qg.hpp:329-335): accept if rp holds
// fewer than ef or lowerBound > distance. Here the warp decides all of them
// at once from one count: candidate j is accepted exactly when fewer than ef
// values of {accepted before this expansion} + {candidates before j in this
// expansion} are <= its distance y_j. (While rp is not full that count is
// below ef. Once it is full, lowerBound is the ef-th smallest accepted value
// L, and y < L is "fewer than ef accepted values <= y"; an earlier candidate
// that was rejected has a value >= the bound of its time >= the bound of any
// later time, so counting it changes no decision, and an earlier accepted one
// counts as it should.) The accepted distances before the expansion that can
// count sit in the sorted pool, so the count is a binary search there plus a
// prefix count over the expansion's candidates. The accepted ones are merged
// into the sorted pool in one step, the bound after each of them is read off
// the merged pool (after the t-th of m accepted it is the value at position
// ef - 1 + m - t once rp is full: the later accepted values are all below
// it), and they enter the search pool in list order.
//
// When the output does not depend on how equal distances sit in rp, the warp
// writes it from the sorted pool; otherwise it replays the log on a result
// heap laid out as libstdc++ leaves it, in its own shared memory (the visited
// cache, candidates, search heap and sorted pool are free by then), checking
// every acceptance against the reference's test and every logged bound
// against rp.top() (replay_result, heap_ops.cuh).
//
// Visited set: the direct-mapped cache of evaluated ids in shared memory. It
// may forget an id, never invents one. A forgotten node that is evaluated
// again has its old distance; if it passes the bound now it was accepted
// before and is still in the sorted pool with the same id and distance, and
// it is dropped there.
//
// Lazy mode (ReplayArgs::lazy) keeps no search heap while the smallest
// unpopped distance is unique (the heap's top is then the sorted pool's first
// unpopped entry) and rebuilds it from the logs at the first tie (below).
//
// A query whose search pool, sorted pool or log outgrows its capacity goes to
// the exact global-memory kernel through the spill list.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>

#include "heap_ops.cuh"
#include "lqg_internal.h"
#include "lqg_kernels.cuh"
#include "sq8_batch.cuh"

namespace lqg {

__host__ __device__ inline size_t batch_warp_bytes(uint32_t dim, uint32_t vbits, uint32_t scap,
                                                   uint32_t acap) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 4 * dpad + 4 * ((size_t)1 << vbits) + kCandBytes + 8 * (size_t)scap + 8 * (size_t)acap;
}

// After a search, a warp's visited cache, candidates, search heap and sorted
// pool (contiguous) can hold a result heap of rcap slots.
__host__ __device__ inline bool batch_replays_in_place(uint32_t vbits, uint32_t scap,
                                                       uint32_t acap, uint32_t rcap) {
    return 4 * ((size_t)1 << vbits) + kCandBytes + 8 * (size_t)scap + 8 * (size_t)acap >=
           8 * (size_t)rcap;
}

constexpr uint32_t kPopped = 0x80000000u;  // sorted-pool id flag (ids are < 2^31)

// Rebuilds the search heap of a query that ran without it (lazy mode): the
// reference's pushes (every accepted node in order, read from the result log)
// and pops (each after the logged number of pushes) replayed on an empty
// heap. Every replayed pop must return the node the lazy search popped there.
// Returns false, with the heap unusable, when one does not or the heap would
// outgrow its slots.
__device__ __forceinline__ bool rebuild_search_heap(const heapops::HeapView sp, uint32_t& sn,
                                                    uint32_t sp_max, const uint4* rlog,
                                                    const uint2* plog, uint32_t acc_n,
                                                    uint32_t pops, int lane) {
    using namespace heapops;
    sn = 0;
    uint32_t i = 0;
    for (uint32_t j = 0; j <= pops; ++j) {
        const uint2 pj = j < pops ? plog[j] : make_uint2(acc_n, kNoId);
        while (i < pj.x) {
            const uint32_t cnt = min(32u, pj.x - i);
            if (sn + cnt > sp_max) return false;
            const uint4 e = (uint32_t)lane < cnt ? rlog[i + lane] : make_uint4(0, 0, 0, 0);
            for (uint32_t t = 0; t < cnt; ++t) {
                const uint32_t id = __shfl_sync(kFull, e.x, t);
                const uint32_t yb = __shfl_sync(kFull, e.y, t);
                warp_push(sp, sn, make_uint2(id, yb ^ 0x80000000u), lane);  // -distance
            }
            i += cnt;
        }
        if (j < pops) {
            if (sn == 0 || sp.get(0).x != pj.y) return false;
            warp_pop(sp, sn, lane);
        }
    }
    return true;
}

// Number of entries of the sorted values a[0, n) that are <= y.
__device__ __forceinline__ uint32_t upper_rank(const float* a, uint32_t n, float y) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= y)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Code words in flight per lane in the distance batches (LW). Up to 256
// dimensions, 16 keeps the kernel within its 96 registers without spills at
// degree 32 (32 spilled and ran 13% slower) and larger degrees, which hold
// more neighbour ids, take 8. Longer rows take 32: a 960-byte row fetched 8
// words at a time needs dozens of dependent rounds, which costs more than the
// spills.
constexpr int batch_load_words(int degw) { return degw == 1 ? 16 : 8; }

// Named barriers of the query-per-block form (barrier 0 is __syncthreads).
__device__ __forceinline__ void named_bar(uint32_t id, uint32_t threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}
constexpr uint32_t kCtaStop = 0xFFFFFFFFu;

// H = 0: one warp per query, blocks of up to 5 query warps. H > 0: one query
// per block of 1 + H warps (the latency form for small batches): warp 0 runs
// the search as above, and each expansion's distances are split over all the
// block's warps, 32 / (H + 1) candidates each, one round of code loads for
// rows of up to 128 bytes; the other warps only compute distances.
template <int G, int DEGW, int LW, int H = 0>
__global__ void __launch_bounds__(H ? 32 * (H + 1) : 160, 4)
    batch_search_kernel(SearchArgs a, ReplayArgs ra) {
    static_assert(H == 0 || (32 / G) * (H + 1) == 32, "helpers split 32 candidates");
    using namespace heapops;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = H ? 0 : (int)(threadIdx.x >> 5);  // the warp's search area
    const int hw = (int)(threadIdx.x >> 5);            // H > 0: 0 searches, others help
    const uint32_t dim = a.dim;
    const uint32_t dpad = (dim + 15u) & ~15u;
    float* pmin = reinterpret_cast<float*>(smem);
    float* pscale = pmin + dpad;
    const uint32_t vbits = a.vbits;
    const uint32_t vsize = 1u << vbits;
    const uint32_t acap = ra.acap;
    unsigned char* wb =
        smem + 8u * dpad + (size_t)warp * batch_warp_bytes(dim, vbits, ra.scap, acap);
    float* qs = reinterpret_cast<float*>(wb);
    uint32_t* vis = reinterpret_cast<uint32_t*>(wb + 4u * dpad);
    uint32_t* cid = vis + vsize;
    float* cd = reinterpret_cast<float*>(cid + kMaxDeg);
    uint2* sps = reinterpret_cast<uint2*>(cd + kMaxDeg);
    float* ad = reinterpret_cast<float*>(sps + ra.scap);  // sorted pool: distances
    uint32_t* ai = reinterpret_cast<uint32_t*>(ad + acap);  // and ids
    const size_t gw = (size_t)blockIdx.x * (H ? 1u : (blockDim.x >> 5)) + warp;
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
    __shared__ uint32_t s_cmd;   // H > 0: candidates to evaluate, or kCtaStop
    __shared__ uint32_t s_hint;  // H > 0: the first unpopped pool entry's id
    constexpr uint32_t kCtaThreads = 32u * (H + 1);
    if constexpr (H > 0) {
        if (hw > 0) {
            for (;;) {
                named_bar(1, kCtaThreads);
                const uint32_t nc = s_cmd;
                if (nc == kCtaStop) break;
                const uint32_t hint = s_hint;
                for (uint32_t b = 0; b < nc; b += 32)
                    eval_batch<G, 1, LW, 1>(a, cid, cd, b + (uint32_t)hw * (32 / G), nc, qs, pmin,
                                            pscale, g, r);
                // The next pop is the first unpopped pool entry or, if one of
                // this expansion's candidates is accepted below it, that one.
                // While warp 0 merges, warp 1 reads the pool entry's neighbour
                // list and asks L2 for their code rows, warp 2 the same for the
                // nearest candidate. Hints only: the ids are clamped to the
                // index, and a wrong guess costs L2 traffic, not results.
                named_bar(2, kCtaThreads);  // every distance is in cd from here
                uint32_t node = kNoId;
                if (hw == 1) {
                    node = hint;
                } else if (hw == 2 && nc > 0) {
                    float best = INF;
                    uint32_t bi = 0;
                    for (uint32_t c = lane; c < nc; c += 32)
                        if (cd[c] < best) {
                            best = cd[c];
                            bi = c;
                        }
#pragma unroll
                    for (int o = 16; o; o >>= 1) {
                        const float ob = __shfl_xor_sync(kFull, best, o);
                        const uint32_t oi = __shfl_xor_sync(kFull, bi, o);
                        if (ob < best || (ob == best && oi < bi)) {
                            best = ob;
                            bi = oi;
                        }
                    }
                    node = cid[bi];
                }
                if (node != kNoId) {
                    node = min(node, a.n - 1u);
                    const uint32_t* nb = a.nbrs + (size_t)node * a.deg;
                    for (uint32_t j = lane; j < a.deg; j += 32) {
                        const uint32_t v = min(__ldg(nb + j), a.n - 1u);
                        const unsigned char* row = a.codes + (size_t)v * a.cstride;
                        for (uint32_t off = 0; off < dim; off += 128)
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(row + off));
                    }
                }
            }
            return;
        }
    }
    // distances of cid[0, nc) into cd: this warp alone, or split over the block
    auto eval_all = [&](uint32_t nc, uint32_t hint) {
        if constexpr (H > 0) {
            if (lane == 0) {
                s_cmd = nc;
                s_hint = hint;
            }
            __syncwarp();
            named_bar(1, kCtaThreads);
            for (uint32_t b = 0; b < nc; b += 32)
                eval_batch<G, 1, LW, 1>(a, cid, cd, b, nc, qs, pmin, pscale, g, r);
            named_bar(2, kCtaThreads);
        } else {
            for (uint32_t b = 0; b < nc; b += 32)
                eval_batch<G, G, LW, 1>(a, cid, cd, b, nc, qs, pmin, pscale, g, r);
        }
    };

    for (;;) {
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(a.qhead, 1u);
        slot = __shfl_sync(kFull, slot, 0);
        if ((int64_t)slot >= mlist) break;
        const int64_t qi = a.qlist ? (int64_t)a.qlist[slot] : (int64_t)slot;
        uint32_t ef = query_ef(a, qi);
        ef = min(max(ef, 1u), ra.efcap);  // efcap <= acap - 32
        const float* q = a.queries + (size_t)qi * dim;
        uint4* rlog = ra.rlog + (size_t)qi * ra.rlog_cap;
        for (uint32_t i = lane; i < dpad; i += 32) qs[i] = i < dim ? q[i] : 0.f;
        for (uint32_t i = lane; i < vsize; i += 32) vis[i] = kNoId;
        __syncwarp();

        // qg.hpp:305-311: the entry point seeds both pools and is visited
        const uint32_t ep = a.entry;
        if (lane == 0) cid[0] = ep;
        __syncwarp();
        if constexpr (H > 0)
            eval_batch<G, 1, LW, 1>(a, cid, cd, 0, 1, qs, pmin, pscale, g, r);
        else
            eval_batch<G, G, LW, 1>(a, cid, cd, 0, 1, qs, pmin, pscale, g, r);
        __syncwarp();
        const float d0 = cd[0];
        bool fail = !(d0 < INF);
        uint32_t acc_n = 1;  // accepted so far (rp.size() = min(acc_n, ef))
        uint32_t alen = 1;   // sorted-pool entries
        float lower = d0;
        uint32_t sn = 1;
        if (lane == 0) {
            sp.set(0, make_uint2(ep, __float_as_uint(-d0)));
            ad[0] = d0;
            ai[0] = ep;
            vis[hash_id(ep, vbits)] = ep;
            rlog[0] = make_uint4(ep, __float_as_uint(d0), __float_as_uint(d0), 0u);
        }
        __syncwarp();
        uint32_t pops = 0, calcs = 1;
        // Lazy mode: no search heap until a pop meets a tie. The heap's live
        // entries (distance <= lowerBound; the others are never popped) are
        // exactly the unpopped entries of the sorted pool, so while the
        // smallest of them is unique it is the heap's top. `cur` is the first
        // unpopped entry; pops are logged (pushes are the result log) so the
        // heap can be rebuilt when the smallest distance is shared.
        bool heap = !ra.lazy;
        uint32_t cur = 0;
        uint2* plg = ra.plog ? ra.plog + (size_t)qi * ra.rlog_cap : nullptr;

        while (!fail) {
            // qg.hpp:313-318
            uint32_t u;
            if (heap) {
                if (sn == 0) break;
                const uint2 top = sp.get(0);
                if (-__uint_as_float(top.y) > lower) break;
                warp_pop(sp, sn, lane);
                u = top.x;
            } else {
                if (cur >= alen) break;  // nothing live: top > lowerBound or empty
                uint32_t nxt = alen;
                for (uint32_t x0 = cur + 1; x0 < alen; x0 += 32) {
                    const uint32_t x = x0 + lane;
                    const unsigned um = __ballot_sync(kFull, x < alen && !(ai[x] & kPopped));
                    if (um) {
                        nxt = x0 + __ffs(um) - 1;
                        break;
                    }
                }
                if (nxt < alen && ad[nxt] == ad[cur]) {
                    // equal smallest distances: the heap layout decides
                    if (!rebuild_search_heap(sp, sn, sp_max, rlog, plg, acc_n, pops, lane)) {
                        fail = true;
                        break;
                    }
                    heap = true;
                    continue;
                }
                if (pops >= ra.rlog_cap) {
                    fail = true;
                    break;
                }
                u = ai[cur];
                __syncwarp();
                if (lane == 0) {
                    ai[cur] = u | kPopped;
                    plg[pops] = make_uint2(acc_n, u);
                }
                __syncwarp();
                cur = nxt;
            }
            ++pops;

            // qg.hpp:320-324: unvisited neighbours in list order
            uint32_t ncand = 0;
            const uint32_t* nb = a.nbrs + (size_t)u * a.deg;
            uint32_t v[DEGW];
#pragma unroll
            for (int w = 0; w < DEGW; ++w) v[w] = __ldg(nb + w * 32 + lane);
            // A list of degree > 32 spans DEGW words. Repeats inside a word
            // are caught by match_any; a repeat of an id kept by an earlier
            // word is caught by the cache, unless another id kept in this
            // expansion took its slot: then (rare) later words also compare
            // against the ids already kept, so no node is a candidate twice
            // (qg.hpp:321). The duplicate check of the acceptance step only
            // sees the pool from before this expansion.
            bool lost = false;
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t h = hash_id(v[w], vbits);
                const bool seen = vis[h] == v[w];
                const unsigned mm = __match_any_sync(kFull, v[w]);
                bool keep = !seen && (mm & lt) == 0;
                if (DEGW > 1 && w > 0 && lost && keep)
                    for (uint32_t j = 0; j < ncand; ++j)
                        if (cid[j] == v[w]) {
                            keep = false;
                            break;
                        }
                __syncwarp();
                if (keep) vis[h] = v[w];
                const unsigned kb = __ballot_sync(kFull, keep);
                if (keep) cid[ncand + __popc(kb & lt)] = v[w];
                ncand += __popc(kb);
                __syncwarp();
                if (DEGW > 1 && w + 1 < DEGW) lost = lost || __any_sync(kFull, keep && vis[h] != v[w]);
            }

            // qg.hpp:325-328
            if constexpr (H > 0) {
                // the next pop is the first unpopped pool entry or an accepted
                // candidate of this expansion: ask L2 for the pool entry's list
                // while the distances are computed
                if (cur < alen && lane == 0)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.nbrs + (size_t)(ai[cur] & ~kPopped) *
                                                                         a.deg));
            }
            eval_all(ncand, cur < alen ? (ai[cur] & ~kPopped) : kNoId);
            calcs += ncand;
            __syncwarp();

            // qg.hpp:329-335: 32 candidates of the list at a time, in order
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t c0 = w * 32;
                if (c0 >= ncand) break;
                const uint32_t c = c0 + lane;
                const bool valid = c < ncand;
                const float y = valid ? cd[c] : INF;
                const uint32_t id = valid ? cid[c] : kNoId;
                if (__any_sync(kFull, valid && !(y < INF))) {
                    fail = true;
                    break;
                }
                // members: candidates that can pass (all while rp is not full)
                bool mem = valid && (acc_n < ef || y < lower);
                uint32_t ub = 0;
                if (mem) {
                    ub = upper_rank(ad, alen, y);
                    // a node the visited cache forgot: still pooled, same distance
                    for (uint32_t x = ub; x > 0 && ad[x - 1] == y; --x)
                        if ((ai[x - 1] & ~kPopped) == id) {
                            mem = false;
                            break;
                        }
                }
                const unsigned mmask = __ballot_sync(kFull, mem);
                if (mmask == 0) continue;
                // earlier members at or below y
                uint32_t pc = 0;
                {
                    unsigned bm = mmask;
                    while (bm) {
                        const int s = __ffs(bm) - 1;
                        bm &= bm - 1;
                        const float ys = __shfl_sync(kFull, y, s);
                        pc += (s < lane && ys <= y) ? 1u : 0u;
                    }
                }
                const bool acc = mem && ub + pc < ef;
                const unsigned am = __ballot_sync(kFull, acc);
                const uint32_t m = __popc(am);
                if (m == 0) continue;
                if (alen + m > acap || acc_n + m > ra.rlog_cap || (heap && sn + m > sp_max)) {
                    fail = true;
                    break;
                }
                // merge: accepted j goes after the pooled values <= y_j and the
                // accepted ones below it (equal ones in list order); pooled
                // entry x moves up by the number of accepted j with ub_j <= x
                uint32_t before = 0;
                uint32_t ubmin = acap;
                uint32_t shc = 0;   // lazy: accepted ones that go before entry `cur`
                float pmax = -INF;  // largest accepted value up to this lane
                {
                    unsigned bm = am;
                    while (bm) {
                        const int s = __ffs(bm) - 1;
                        bm &= bm - 1;
                        const float ys = __shfl_sync(kFull, y, s);
                        const uint32_t us = __shfl_sync(kFull, ub, s);
                        before += (ys < y || (ys == y && s < lane)) ? 1u : 0u;
                        ubmin = min(ubmin, us);
                        shc += us <= cur ? 1u : 0u;
                        if (s <= lane) pmax = fmaxf(pmax, ys);
                    }
                }
                const float old_max = ad[alen - 1];
                for (int rr = (int)((alen - 1) >> 5); rr >= (int)(ubmin >> 5); --rr) {
                    const uint32_t x = (uint32_t)rr * 32 + lane;
                    const bool have = x < alen && x >= ubmin;
                    float xd = 0.f;
                    uint32_t xi = 0;
                    if (have) {
                        xd = ad[x];
                        xi = ai[x];
                    }
                    uint32_t sh = 0;
                    unsigned bm = am;
                    while (bm) {
                        const int s = __ffs(bm) - 1;
                        bm &= bm - 1;
                        sh += __shfl_sync(kFull, ub, s) <= x ? 1u : 0u;
                    }
                    __syncwarp();
                    if (have) {
                        ad[x + sh] = xd;
                        ai[x + sh] = xi;
                    }
                    __syncwarp();
                }
                if (acc) {
                    ad[ub + before] = y;
                    ai[ub + before] = id;
                }
                __syncwarp();
                // the first unpopped entry: the one at `cur` moved up, or an
                // accepted one placed before it
                cur = min(cur + shc, __reduce_min_sync(kFull, acc ? ub + before : 0xFFFFFFFFu));
                alen += m;
                const uint32_t acc_new = acc_n + m;
                const float lf = ad[min(acc_new, ef) - 1];
                // the bound after the t-th accepted (qg.hpp:333-334), logged
                const uint32_t t = __popc(am & lt) + 1;
                if (acc) {
                    const float lb = acc_n + t >= ef ? ad[ef - 1 + m - t] : fmaxf(old_max, pmax);
                    rlog[acc_n + t - 1] =
                        make_uint4(id, __float_as_uint(y), __float_as_uint(lb), 0u);
                }
                // rp trims its largest: beyond position ef only ties with the
                // bound stay in the sorted pool
                if (acc_new > ef) {
                    uint32_t keep = ef;
                    for (uint32_t x0 = ef; x0 < alen; x0 += 32) {
                        const uint32_t x = x0 + lane;
                        const unsigned em = __ballot_sync(kFull, x < alen && ad[x] == lf);
                        keep += __popc(em);
                        if (em != kFull) break;
                    }
                    alen = keep;
                }
                lower = lf;
                acc_n = acc_new;
                // the search pool takes them in list order (qg.hpp:332)
                unsigned bm = heap ? am : 0u;
                while (bm) {
                    const int s = __ffs(bm) - 1;
                    bm &= bm - 1;
                    const uint32_t sid = __shfl_sync(kFull, id, s);
                    const float ys = __shfl_sync(kFull, y, s);
                    warp_push(sp, sn, make_uint2(sid, __float_as_uint(-ys)), lane);
                }
                __syncwarp();
            }
        }

        // Output (qg.hpp:340-343). rp pops come out in descending distance;
        // only equal distances make the heap layout decide. So when the
        // sorted pool holds exactly rp (no ties beyond the ef-th entry) and
        // the popped entries (the worst k and the one after them, or the
        // whole pool when it is returned) have distinct distances, the output
        // is read off the pool; otherwise the log is replayed.
        const uint32_t P = min(acc_n, ef);
        bool direct = false;
        if (!fail && !ra.replay_all) {
            const uint32_t k = min(a.kq ? a.kq[qi] : a.k0, a.kstride);
            const uint32_t kk = min(k, P);
            const uint32_t lo = a.pool_ids ? 0u : (P > kk ? P - kk - 1 : 0u);
            bool tie = false;
            for (uint32_t x = lo + lane; x + 1 < P; x += 32) tie |= ad[x] == ad[x + 1];
            direct = alen == P && !__any_sync(kFull, tie);
            if (direct) {
                uint32_t* out = a.ids + (size_t)qi * a.kstride;
                for (uint32_t x = lane; x < k - kk; x += 32) out[x] = kNoId;
                for (uint32_t x = P - kk + lane; x < P; x += 32)
                    out[x + k - P] = ai[x] & ~kPopped;
                if (a.pool_ids) {
                    for (uint32_t x = lane; x < a.pstride; x += 32) {
                        a.pool_ids[(size_t)qi * a.pstride + x] = x < P ? ai[x] & ~kPopped : kNoId;
                        a.pool_d[(size_t)qi * a.pstride + x] = x < P ? ad[x] : INF;
                    }
                }
            }
        }
        if (!fail && !direct && !ra.replay_all &&
            batch_replays_in_place(vbits, ra.scap, acap, ra.rcap)) {
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
    if constexpr (H > 0) {
        if (lane == 0) s_cmd = kCtaStop;
        __syncwarp();
        named_bar(1, kCtaThreads);
    }
}

template <int G, int DEGW, int LW, int H = 0>
static cudaError_t batch_run(const SearchArgs& a, const ReplayArgs& ra, int warps, int blocks,
                            cudaStream_t st, int* occ) {
    const size_t dpad = (a.dim + 15u) & ~15u;
    const int areas = H ? 1 : warps;
    const int threads = H ? 32 * (H + 1) : warps * 32;
    const size_t smem = 8 * dpad + (size_t)areas * batch_warp_bytes(a.dim, a.vbits, ra.scap, ra.acap);
    auto k = batch_search_kernel<G, DEGW, LW, H>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, threads, smem);
    k<<<blocks, threads, smem, st>>>(a, ra);
    return cudaGetLastError();
}

// The query-per-block form: 4 lanes per candidate, 4 warps (8 candidates
// each); a lane holds one code word per 16-dimension chunk, so 16 words in
// flight cover 8 chunks per round.
template <int DEGW>
cudaError_t batch_cta_run(const SearchArgs& a, const ReplayArgs& ra, int blocks, cudaStream_t st,
                          int* occ) {
    return batch_run<4, DEGW, 16, 3>(a, ra, 1, blocks, st, occ);
}

// All instances for one lanes-per-candidate G: degree words 1-4, each with
// the short and the long code-load window.
template <int G>
cudaError_t batch_dispatch(const SearchArgs& a, const ReplayArgs& ra, int degw, int warps,
                           int blocks, cudaStream_t st, int* occ) {
    const bool wide = a.dim >= kBatchWideDim;
#define LQG_BCASE(DW)                                                                   \
    case DW:                                                                            \
        return wide ? batch_run<G, DW, 32>(a, ra, warps, blocks, st, occ)               \
                    : batch_run<G, DW, batch_load_words(DW)>(a, ra, warps, blocks, st, occ);
    switch (degw) {
        LQG_BCASE(1)
        LQG_BCASE(2)
        LQG_BCASE(3)
        LQG_BCASE(4)
        default: return cudaErrorInvalidValue;
    }
#undef LQG_BCASE
}

}  // namespace lqg
