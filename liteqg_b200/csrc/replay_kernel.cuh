// Replay search: the reference's search loop (QuantizedGraph::
// search_qg_with_heap, symqglib/qg/qg.hpp:298-344), exact for every query,
// ties included, with the libstdc++ heap work taken off the search's critical
// path. Two kernels:
//
// replay_search_kernel: a block holds S search warps (one query each,
// persistent over the work queue) and one replay warp whose lane j runs the
// reference's search pool (a std::priority_queue) for search warp j.
//
// Search warp. It needs only three things from the pools, and none of them
// depends on how equal distances sit in the heaps:
//   * rp.size() = min(accepted, ef);
//   * lowerBound = rp.top().distance = the ef-th smallest accepted distance
//     (each trim removes a largest element, so rp's multiset of distances is
//     the ef smallest accepted ones), or the largest one while rp is not full;
//   * the next pop: sp holds every accepted node not yet popped. One with a
//     distance above lowerBound never pops again (the bound only falls once
//     rp is full). So the nodes that can pop are exactly the accepted,
//     unpopped nodes at or below the bound, and the search warp keeps all
//     accepted nodes at or below the bound in a sorted register array
//     (E entries per lane, "popped" flag in bit 31 of the id). The smallest
//     unpopped entry is sp.top() unless another unpopped entry has the same
//     distance; only then does the heap layout decide, and the warp asks the
//     replay lane for sp.top().
// Neighbours are accepted in list order against the current size and bound
// (qg.hpp:329-335). The search-pool operations go to a per-warp log ring in
// shared memory (PUSH(id, dist), POP(id), BEGIN(query), END(bound)); every
// accepted node also goes to the query's result log in global memory
// (id, dist, bound after).
//
// Replay lane. It replays the ring on a search heap laid out exactly as GCC
// libstdc++'s push_heap/pop_heap leave it (bits/stl_heap.h: push = sift-up
// while comp(parent, value); pop = hole from the root to a leaf along the
// larger child, the right one unless comp(right, left), then sift-up of the
// last element), checks that each POP is sp.top() and that at END the
// reference's loop would stop, and answers the tie questions.
//
// rp_replay_kernel (one warp per query, after the search): replays the
// result log on a result heap laid out as libstdc++ leaves it, checks each
// accepted node against the reference's acceptance test on that heap and the
// logged bound against rp.top(), and writes the output by popping rp
// (qg.hpp:340-343).
//
// A query that fails a check, or outgrows a pool or its log, goes to the exact
// global-memory kernel through the spill list.
//
// Visited set: a direct-mapped cache of evaluated ids in shared memory. It may
// forget an id, never invents one. A forgotten node that is evaluated again
// has its old distance; if it passes the acceptance test now, it was accepted
// before and is still in the register array (at or below the bound) with the
// same id and distance, and it is dropped there. So the accepted sequence is
// the reference's.
//
// Distances: G lanes per candidate, 32/G candidates per pass, all passes'
// code bytes requested before any arithmetic; decode and L2 with the packed
// f32x2 instructions (two IEEE round-to-nearest FP32 operations each, the same
// bits as the scalar ones) in the reference's 16-accumulator order.
#pragma once
#include <cuda/atomic>
#include <cuda_runtime.h>
#include <math_constants.h>

#include "lqg_internal.h"
#include "lqg_kernels.cuh"
#include "sq8_batch.cuh"

namespace lqg {

namespace replay {

constexpr uint32_t kLogN = kReplayLogN;
// Markers in the distance word of a log entry: non-finite patterns that a
// finite, non-negative distance never has.
constexpr uint32_t kOpPop = 0xFFFFFFF0u;
constexpr uint32_t kOpBegin = 0xFFFFFFF1u;
constexpr uint32_t kOpEnd = 0xFFFFFFF2u;
constexpr uint32_t kOpEndFail = 0xFFFFFFF3u;
constexpr uint32_t kOpFinish = 0xFFFFFFF4u;
// Spin limit (iterations of about 100 ns): a wait that runs out sets
// kErrSync and the block returns.
constexpr uint32_t kSpinLimit = 1u << 24;

struct Ctl {
    uint32_t head;  // ring entries written (search warp)
    uint32_t tail;  // ring entries replayed (replay lane)
    uint32_t pad0, pad1;
};

__device__ __forceinline__ uint32_t load_acq(uint32_t* p) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_block> r(*p);
    return r.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void store_rel(uint32_t* p, uint32_t v) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_block> r(*p);
    r.store(v, cuda::memory_order_release);
}
__device__ __forceinline__ uint32_t load_rlx(uint32_t* p) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_block> r(*p);
    return r.load(cuda::memory_order_relaxed);
}

// ---- heaps (one lane) ------------------------------------------------------

__device__ __forceinline__ uint2 lds2(uint32_t addr) {
    uint2 v;
    asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ void sts2(uint32_t addr, uint2 v) {
    asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(addr), "r"(v.x), "r"(v.y) : "memory");
}

// A heap array: slots [0, cap) in shared memory (32-bit shared address s),
// slots >= cap in a global-memory area g.
struct Heap {
    uint32_t s;
    uint2* g;
    uint32_t cap;
    __device__ __forceinline__ uint2 get(uint32_t i) const {
        return i < cap ? lds2(s + 8u * i) : g[i - cap];
    }
    __device__ __forceinline__ void set(uint32_t i, uint2 v) const {
        if (i < cap)
            sts2(s + 8u * i, v);
        else
            g[i - cap] = v;
    }
};

__device__ __forceinline__ float hkey(uint2 x) { return __uint_as_float(x.y); }

// libstdc++ __push_heap(first, hole, 0, v): sift v up from `hole`.
__device__ __forceinline__ void sift_up(const Heap& h, uint32_t hole, uint2 v) {
    while (hole > 0) {
        const uint32_t parent = (hole - 1) / 2;
        const uint2 p = h.get(parent);
        if (!(hkey(p) < hkey(v))) break;
        h.set(hole, p);
        hole = parent;
    }
    h.set(hole, v);
}

// pop_heap over [0, n) (the caller then drops slot n - 1): libstdc++
// __pop_heap + __adjust_heap with top index 0.
__device__ __forceinline__ void pop_top(const Heap& h, uint32_t n) {
    if (n <= 1) return;
    const uint32_t len = n - 1;
    const uint2 v = h.get(len);
    uint32_t hole = 0, second = 0;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        const uint2 r = h.get(second);
        const uint2 l = h.get(second - 1);
        if (hkey(r) < hkey(l)) {
            --second;
            h.set(hole, l);
        } else {
            h.set(hole, r);
        }
        hole = second;
    }
    if ((len & 1u) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        h.set(hole, h.get(second - 1));
        hole = second - 1;
    }
    sift_up(h, hole, v);
}

}  // namespace replay

template <int E>
__device__ __forceinline__ float rpool_at(const float (&pd)[E], uint32_t pos) {
    const uint32_t l = pos / E, s = pos % E;
    float v = pd[0];
#pragma unroll
    for (int t = 1; t < E; ++t)
        if (s == (uint32_t)t) v = pd[t];
    return __shfl_sync(kFull, v, l);
}

template <int E, int G, int DEGW>
__global__ void __launch_bounds__(512) replay_search_kernel(SearchArgs a, ReplayArgs ra) {
    using namespace replay;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t S = ra.swarps;
    const uint32_t dim = a.dim;
    const uint32_t dpad = (dim + 15u) & ~15u;
    float* pmin = reinterpret_cast<float*>(smem);
    float* pscale = pmin + dpad;
    const uint32_t vbits = a.vbits;
    const uint32_t vsize = 1u << vbits;
    const size_t wbytes = replay_warp_bytes(dim, vbits, ra.scap);
    unsigned char* const base0 = smem + 8u * dpad;

    for (uint32_t i = threadIdx.x; i < dpad; i += blockDim.x) {
        pmin[i] = i < dim ? a.params[2 * i] : 0.f;
        pscale[i] = i < dim ? a.params[2 * i + 1] : 0.f;
    }
    if ((uint32_t)warp < S && lane == 0) {
        Ctl* c = reinterpret_cast<Ctl*>(base0 + (size_t)warp * wbytes + wbytes - sizeof(Ctl));
        c->head = 0;
        c->tail = 0;
    }
    __shared__ uint32_t block_abort;
    if (threadIdx.x == 0) block_abort = 0;
    __syncthreads();

    // per-warp region: query | visited cache | candidates | ring | sp | ctl
    auto region = [&](uint32_t j) { return base0 + (size_t)j * wbytes; };
    auto ring_of = [&](unsigned char* wb) {
        return reinterpret_cast<uint2*>(wb + 4u * dpad + 4u * vsize + kCandBytes);
    };
    auto sp_of = [&](unsigned char* wb) {
        return reinterpret_cast<uint2*>(wb + 4u * dpad + 4u * vsize + kCandBytes + 8u * kLogN);
    };

    if ((uint32_t)warp == S) {
        // ====== replay warp: lane j runs search warp j's search heap ======
        const uint32_t j = (uint32_t)lane;
        bool fin = j >= S;
        unsigned char* wb = region(fin ? 0u : j);
        const uint2* ring = ring_of(wb);
        Ctl* ctl = reinterpret_cast<Ctl*>(wb + wbytes - sizeof(Ctl));
        const size_t gw = (size_t)blockIdx.x * S + j;
        const Heap sp{(uint32_t)__cvta_generic_to_shared(sp_of(wb)),
                      ra.sp_global + (fin ? 0 : gw) * ra.gcap, ra.scap};
        const uint32_t sp_max = ra.scap + ra.gcap;
        uint32_t tail = 0, released = 0, head_c = 0;
        int64_t qi = 0;
        uint32_t n = 0;
        bool err = false;
        uint32_t idle = 0;
        auto spill = [&]() {
            const uint32_t i = atomicAdd(ra.nspill, 1u);
            ra.spill[i] = (int32_t)qi;
            ra.rlen[qi] = kNoId;  // the result pass skips it
        };
        for (;;) {
            bool progressed = false, dopop = false;
            uint32_t pn = 0;
            if (!fin) {
                if (tail == head_c) head_c = load_acq(&ctl->head);
                if (tail != head_c) {
                    const uint2 e = ring[tail % kLogN];
                    ++tail;
                    progressed = true;
                    if (e.y == kOpBegin) {
                        qi = (int64_t)e.x;
                        n = 0;
                        err = false;
                    } else if (e.y == kOpPop) {
                        // qg.hpp:314-318: the search warp popped sp.top()
                        if (!err) {
                            if (n == 0 || sp.get(0).x != e.x) {
                                err = true;
                            } else {
                                dopop = true;
                                pn = n;
                                --n;
                            }
                        }
                    } else if (e.y == kOpEnd) {
                        // the reference's loop stops here: sp empty or its top above the bound
                        const bool ok = !err && (n == 0 || -hkey(sp.get(0)) > __uint_as_float(e.x));
                        if (!ok) spill();
                    } else if (e.y == kOpEndFail) {
                        spill();
                    } else if (e.y == kOpFinish) {
                        fin = true;
                    } else if (!err) {
                        // PUSH (qg.hpp:330)
                        if (n >= sp_max) {
                            err = true;
                        } else {
                            sift_up(sp, n, make_uint2(e.x, __float_as_uint(-__uint_as_float(e.y))));
                            ++n;
                        }
                    }
                }
            }
            if (dopop) pop_top(sp, pn);
            // publish progress when caught up, or every 16 entries
            if (j < S && tail != released && (tail == head_c || tail - released >= 16 || fin)) {
                store_rel(&ctl->tail, tail);
                released = tail;
            }
            if (!__ballot_sync(kFull, !fin)) break;
            if (!__ballot_sync(kFull, progressed)) {
                if (__any_sync(kFull, load_rlx(&block_abort) != 0u)) break;
                if (++idle > kSpinLimit) {
                    atomicOr(a.err, kErrSync);
                    atomicExch(&block_abort, 1u);
                    break;
                }
                __nanosleep(64);
            } else {
                idle = 0;
            }
        }
        return;
    }

    // ======================= search warp =======================
    unsigned char* wb = region((uint32_t)warp);
    float* qs = reinterpret_cast<float*>(wb);
    uint32_t* vis = reinterpret_cast<uint32_t*>(wb + 4u * dpad);
    uint32_t* cid = vis + vsize;
    float* cd = reinterpret_cast<float*>(cid + kMaxDeg);
    uint2* ring = ring_of(wb);
    const uint2* sp_top = sp_of(wb);
    Ctl* ctl = reinterpret_cast<Ctl*>(wb + wbytes - sizeof(Ctl));

    const int g = lane / G, r = lane % G;
    const uint32_t lt = lanemask_lt();
    const int64_t mlist = a.nlist ? (int64_t)*a.nlist : a.m;
    const float INF = CUDART_INF_F;
    constexpr uint32_t CAP = 32u * E;
    constexpr int NP = G;  // passes per distance batch: 32 candidates
    constexpr uint32_t BATCH = (uint32_t)NP * (32 / G);

    // ring writer state (lane 0)
    uint32_t head = 0, tail_c = 0;
    bool aborted = false;
    auto publish = [&]() {
        if (lane == 0) store_rel(&ctl->head, head);
    };
    // lane 0 appends one ring entry; waits (bounded) for room
    auto put = [&](uint2 e) {
        if (lane == 0 && !aborted) {
            if (head - tail_c >= kLogN) {
                store_rel(&ctl->head, head);
                uint32_t spin = 0;
                while (head - (tail_c = load_acq(&ctl->tail)) >= kLogN) {
                    if (++spin > kSpinLimit || load_rlx(&block_abort)) {
                        atomicOr(a.err, kErrSync);
                        atomicExch(&block_abort, 1u);
                        aborted = true;
                        break;
                    }
                    __nanosleep(100);
                }
            }
            if (!aborted) {
                ring[head % kLogN] = e;
                ++head;
            }
        }
    };

    for (;;) {
        uint32_t slot = 0;
        if (lane == 0) slot = aborted ? 0xFFFFFFFFu : atomicAdd(a.qhead, 1u);
        slot = __shfl_sync(kFull, slot, 0);
        if ((int64_t)slot >= mlist || slot == 0xFFFFFFFFu) break;
        const int64_t qi = a.qlist ? (int64_t)a.qlist[slot] : (int64_t)slot;
        uint32_t ef = query_ef(a, qi);
        ef = min(max(ef, 1u), ra.efcap);  // efcap <= CAP - 32
        const float* q = a.queries + (size_t)qi * dim;
        uint4* rlog = ra.rlog + (size_t)qi * ra.rlog_cap;
        for (uint32_t i = lane; i < dpad; i += 32) qs[i] = i < dim ? q[i] : 0.f;
        for (uint32_t i = lane; i < vsize; i += 32) vis[i] = kNoId;
        put(make_uint2((uint32_t)qi, kOpBegin));
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
        eval_batch<G, NP>(a, cid, cd, 0, 1, qs, pmin, pscale, g, r);
        __syncwarp();
        const float d0 = cd[0];
        bool fail = !(d0 < INF);
        uint32_t acc_n = 1;  // accepted so far (rp.size() = min(acc_n, ef))
        float lower = d0;
        if (lane == 0) {
            pd[0] = d0;
            pi[0] = ep;
            vis[hash_id(ep, vbits)] = ep;
            rlog[0] = make_uint4(ep, __float_as_uint(d0), __float_as_uint(d0), 0u);
        }
        put(make_uint2(ep, __float_as_uint(d0)));
        __syncwarp();
        uint32_t pops = 0, calcs = 1;

        while (!fail) {
            // ---- qg.hpp:313-318: the next pop ----
            int tf = E;
#pragma unroll
            for (int t = E - 1; t >= 0; --t)
                if (!(pi[t] & kExpanded)) tf = t;
            const unsigned hb = __ballot_sync(kFull, tf < E);
            if (!hb) break;  // every node at or below the bound has popped: sp.top() > bound
            const int owner = __ffs(hb) - 1;
            float mine = 0.f;
#pragma unroll
            for (int t = 0; t < E; ++t)
                if (t == tf) mine = pd[t];
            const float dmin = __shfl_sync(kFull, mine, owner);
            uint32_t cnt = 0;
#pragma unroll
            for (int t = 0; t < E; ++t) cnt += (!(pi[t] & kExpanded) && pd[t] == dmin) ? 1u : 0u;
            const uint32_t nt = __reduce_add_sync(kFull, cnt);
            uint32_t u;
            if (nt == 1) {
                uint32_t mu = 0;
                if (lane == owner) {
#pragma unroll
                    for (int t = 0; t < E; ++t)
                        if (t == tf) {
                            mu = pi[t];
                            pi[t] |= kExpanded;
                        }
                }
                u = __shfl_sync(kFull, mu, owner);
            } else {
                // equal distances: the heap layout decides; ask the replay lane
                uint32_t top = kNoId;
                if (lane == 0 && !aborted) {
                    store_rel(&ctl->head, head);
                    uint32_t spin = 0;
                    while (load_acq(&ctl->tail) != head) {
                        if (++spin > kSpinLimit || load_rlx(&block_abort)) {
                            atomicOr(a.err, kErrSync);
                            atomicExch(&block_abort, 1u);
                            aborted = true;
                            break;
                        }
                        __nanosleep(32);
                    }
                    tail_c = head;
                    if (!aborted) top = sp_top[0].x;
                }
                u = __shfl_sync(kFull, top, 0);
                bool found = false;
#pragma unroll
                for (int t = 0; t < E; ++t)
                    if (pi[t] == u && pd[t] == dmin) {
                        pi[t] |= kExpanded;
                        found = true;
                    }
                if (!__any_sync(kFull, found)) {
                    fail = true;
                    break;
                }
            }
            put(make_uint2(u, kOpPop));
            ++pops;

            // ---- qg.hpp:320-324: unvisited neighbours in list order ----
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

            // ---- qg.hpp:325-328: SQ8 decode + L2 ----
            for (uint32_t b = 0; b < ncand; b += BATCH)
                eval_batch<G, NP>(a, cid, cd, b, ncand, qs, pmin, pscale, g, r);
            calcs += ncand;
            __syncwarp();

            // ---- qg.hpp:329-335: acceptance in list order ----
            const bool full0 = acc_n >= ef;
            const float lower0 = lower;
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t c0 = w * 32;
                if (c0 >= ncand) break;
                const uint32_t c = c0 + lane;
                const float dc = c < ncand ? cd[c] : 0.f;
                if (c < ncand && !(dc < INF)) fail = true;
                const bool pass = c < ncand && (!full0 || lower0 > dc);
                if (__any_sync(kFull, fail)) {
                    fail = true;
                    break;
                }
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
                    for (int t = 0; t < E; ++t) dup |= pd[t] == y && (pi[t] & ~kExpanded) == id;
                    if (__any_sync(kFull, dup)) continue;
                    // room for one more entry (ties at the bound can exceed ef), and in the log
                    if (__shfl_sync(kFull, pd[E - 1], 31) < INF || acc_n >= ra.rlog_cap) {
                        fail = true;
                        break;
                    }
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
                    lower = rpool_at<E>(pd, min(acc_n + 1, ef) - 1);
                    if (acc_n + 1 > ef) {
                        // beyond the ef-th entry only ties with the bound stay poppable
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
                    put(make_uint2(id, __float_as_uint(y)));
                }
                if (fail) break;
            }
            publish();
            if (__shfl_sync(kFull, (int)aborted, 0)) fail = true;
        }

        if (lane == 0) ra.rlen[qi] = fail ? kNoId : acc_n;
        put(make_uint2(fail ? 0u : __float_as_uint(lower), fail ? kOpEndFail : kOpEnd));
        publish();
        if (a.stats && lane == 0) {
            const uint32_t P = min(acc_n, ef);
            *reinterpret_cast<uint4*>(a.stats + 4 * (size_t)qi) = make_uint4(pops, calcs, 0u, P);
        }
        __syncwarp();
        if (__shfl_sync(kFull, (int)aborted, 0)) break;
    }
    put(make_uint2(0u, kOpFinish));
    publish();
}

template <int E, int G, int DEGW>
static cudaError_t replay_run(const SearchArgs& a, const ReplayArgs& ra, int blocks,
                             cudaStream_t st, int* occ) {
    const size_t dpad = (a.dim + 15u) & ~15u;
    const size_t smem =
        8 * dpad + (size_t)ra.swarps * replay_warp_bytes(a.dim, a.vbits, ra.scap);
    auto k = replay_search_kernel<E, G, DEGW>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int threads = 32 * ((int)ra.swarps + 1);
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, threads, smem);
    k<<<blocks, threads, smem, st>>>(a, ra);
    return cudaGetLastError();
}

// All instances for one pool size E: lanes per candidate x degree words.
template <int E>
cudaError_t replay_dispatch(const SearchArgs& a, const ReplayArgs& ra, int G, int degw,
                            int blocks, cudaStream_t st, int* occ) {
#define LQG_RCASE(GG, DW) \
    if (G == GG && degw == DW) return replay_run<E, GG, DW>(a, ra, blocks, st, occ);
#define LQG_RCASES(GG) LQG_RCASE(GG, 1) LQG_RCASE(GG, 2) LQG_RCASE(GG, 3) LQG_RCASE(GG, 4)
    LQG_RCASES(2)
    LQG_RCASES(4)
    LQG_RCASES(8)
#undef LQG_RCASES
#undef LQG_RCASE
    return cudaErrorInvalidValue;
}

}  // namespace lqg
