// Warp-cooperative libstdc++ binary-heap steps on (id, distance bits) pairs,
// shared by the heap and split search kernels. comp(x, y) is x.dist < y.dist
// (symqglib/qg/qg.hpp:289-293); the search pool stores -distance.
//   push: sift-up while comp(parent, value) (GCC bits/stl_heap.h
//         __push_heap). The path from the new slot to the root is known and
//         comp(parent, value) is monotone along it, so lane i loads the i-th
//         ancestor, one ballot gives how far the value rises, and the shifted
//         ancestors are written in one step.
//   pop:  move the last element out, walk a hole from the root to a leaf
//         along the larger child (the right one unless comp(right, left)),
//         then sift the moved element up from there (__pop_heap /
//         __adjust_heap). The walk is data dependent and runs on lane 0; the
//         sift-up is the warp-parallel one.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lqg_internal.h"
#include "lqg_kernels.cuh"

namespace lqg {
namespace heapops {

__device__ __forceinline__ bool hless(uint2 x, uint2 y) {
    return __uint_as_float(x.y) < __uint_as_float(y.y);
}

// A heap array: slots [0, cap) in shared memory, slots >= cap (the deepest
// levels of a large search pool) in a per-warp global-memory area.
struct HeapView {
    uint2* s;
    uint2* g;
    uint32_t cap;
    __device__ __forceinline__ uint2 get(uint32_t i) const { return i < cap ? s[i] : g[i - cap]; }
    __device__ __forceinline__ void set(uint32_t i, uint2 v) const {
        if (i < cap)
            s[i] = v;
        else
            g[i - cap] = v;
    }
};

// Sift-up of v from slot `hole` (libstdc++ __push_heap with top 0), all lanes.
__device__ __forceinline__ void warp_sift_up(HeapView h, uint32_t hole, uint2 v, int lane) {
    // ancestors of hole: ((hole + 1) >> i) - 1 for i = 1 .. depth
    const uint32_t p1 = hole + 1;
    const uint32_t depth = 31u - __clz(p1);  // floor(log2(hole + 1))
    bool pred = false;
    uint2 anc = make_uint2(0, 0);
    if (lane >= 1 && (uint32_t)lane <= depth) {
        anc = h.get((p1 >> lane) - 1u);
        pred = hless(anc, v);
    }
    const unsigned m = __ballot_sync(kFull, pred);
    // consecutive trues from level 1 upward: the loop of __push_heap stops
    // at the first parent that is not less than the value
    const uint32_t j = (uint32_t)(__ffs(~(m >> 1)) - 1);
    // level l (1..j): its value moves down to level l - 1
    if (lane >= 1 && (uint32_t)lane <= j) h.set((p1 >> (lane - 1)) - 1u, anc);
    if (lane == 0) h.set((p1 >> j) - 1u, v);
    __syncwarp();
}

__device__ __forceinline__ void warp_push(HeapView h, uint32_t& n, uint2 v, int lane) {
    warp_sift_up(h, n, v, lane);
    ++n;
}

// pop_heap + pop_back. The hole walk of __adjust_heap goes five levels per
// round: lane i (< 31) takes the i-th node, in breadth-first order, of the
// five-level subtree under the hole, loads its two children and decides
// which one the walk would take from it (left only if comp(right, left)) and
// whether the walk continues there (node < (len - 1) / 2). One ballot per
// bit gives the path; each lane on it moves its chosen child up into its
// node. All loads of a round precede its stores and no path node is read
// after it is written, so the moves are the sequential walk's.
__device__ __forceinline__ void warp_pop(HeapView h, uint32_t& n, int lane) {
    const uint32_t size = n;
    if (size > 1) {
        const uint32_t len = size - 1;
        const uint2 v = h.get(len);
        const uint32_t lim = (len - 1) / 2;
        uint32_t hole = 0;
        // BFS index i: depth k = floor(log2(i + 1)), offset i + 1 - 2^k
        const uint32_t k = 31u - __clz((uint32_t)lane + 1u);
        const uint32_t off = (uint32_t)lane + 1u - (1u << k);
        while (hole < lim) {
            const uint32_t node = ((hole + 1u) << k) - 1u + off;
            const bool cont = lane < 31 && node < lim;
            uint2 ch = make_uint2(0, 0);
            bool left = false;
            if (cont) {
                const uint2 r = h.get(2 * node + 2), l = h.get(2 * node + 1);
                left = hless(r, l);
                ch = left ? l : r;
            }
            const unsigned mc = __ballot_sync(kFull, cont);
            const unsigned ml = __ballot_sync(kFull, left);
            uint32_t i = 0, path = 0;
            int steps = 0;
            while (steps < 5 && ((mc >> i) & 1u)) {
                path |= 1u << i;
                i = 2 * i + (((ml >> i) & 1u) ? 1u : 2u);
                ++steps;
            }
            if ((path >> lane) & 1u) h.set(node, ch);
            __syncwarp();
            // the hole moves to BFS index i (depth `steps`) of this subtree
            hole = ((hole + 1u) << steps) - 1u + (i + 1u - (1u << steps));
            if (steps < 5) break;
        }
        if ((len & 1u) == 0 && hole == (len - 2) / 2) {
            const uint2 c = h.get(2 * hole + 1);
            __syncwarp();
            if (lane == 0) h.set(hole, c);
            __syncwarp();
            hole = 2 * hole + 1;
        }
        warp_sift_up(h, hole, v, lane);
    }
    n = size - 1;
}

}  // namespace heapops

// The result pool of query qi replayed from its log (qg.hpp:329-343) on the
// heap rp (one warp): the logged accepted nodes in order, each checked
// against the reference's acceptance test on this heap (size < ef or top >
// distance) and the logged bound after it against rp.top(); then the output:
// the first k pops (results[k-1-j] = j-th pop) and, if asked, the whole pool
// in ascending order. The log is read 32 entries per coalesced load. Returns
// false (nothing written) when a check fails.
__device__ __forceinline__ bool replay_result(const SearchArgs& a, const ReplayArgs& ra,
                                              int64_t qi, uint32_t len, const heapops::HeapView rp,
                                              int lane) {
    using namespace heapops;
    const uint32_t efq = query_ef(a, qi);
    const uint32_t ef = min(max(efq, 1u), ra.efcap);
    const uint32_t k = min(a.kq ? a.kq[qi] : a.k0, a.kstride);
    const uint4* lg = ra.rlog + (size_t)qi * ra.rlog_cap;
    uint32_t n = 0;
    bool ok = len > 0 && len <= ra.rlog_cap;
    for (uint32_t b = 0; ok && b < len; b += 32) {
        const uint4 mine = b + lane < len ? __ldcs(lg + b + lane) : make_uint4(0, 0, 0, 0);
        const uint32_t cnt = min(32u, len - b);
        for (uint32_t j = 0; j < cnt; ++j) {
            const uint32_t id = __shfl_sync(kFull, mine.x, j);
            const uint32_t yb = __shfl_sync(kFull, mine.y, j);
            const uint32_t lb = __shfl_sync(kFull, mine.z, j);
            if (!(n < ef || __uint_as_float(rp.get(0).y) > __uint_as_float(yb))) {
                ok = false;
                break;
            }
            warp_push(rp, n, make_uint2(id, yb), lane);
            if (n > ef) warp_pop(rp, n, lane);
            if (rp.get(0).y != lb) {
                ok = false;
                break;
            }
        }
    }
    if (!ok) return false;
    const uint32_t P = n, kk = min(k, P);
    uint32_t* out = a.ids + (size_t)qi * a.kstride;
    for (uint32_t x = lane; x < k - kk; x += 32) out[x] = kNoId;
    if (a.pool_ids)
        for (uint32_t x = P + lane; x < a.pstride; x += 32) {
            a.pool_ids[(size_t)qi * a.pstride + x] = kNoId;
            a.pool_d[(size_t)qi * a.pstride + x] = __int_as_float(0x7f800000);
        }
    const uint32_t ex = a.pool_ids ? P : kk;
    for (uint32_t j = 0; j < ex; ++j) {
        const uint2 t = rp.get(0);
        if (lane == 0) {
            if (j < kk) out[k - 1 - j] = t.x;
            if (a.pool_ids && P - 1 - j < a.pstride) {
                a.pool_ids[(size_t)qi * a.pstride + (P - 1 - j)] = t.x;
                a.pool_d[(size_t)qi * a.pstride + (P - 1 - j)] = __uint_as_float(t.y);
            }
        }
        warp_pop(rp, n, lane);
    }
    return true;
}

}  // namespace lqg
