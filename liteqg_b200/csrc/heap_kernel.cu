// Heap search kernel: the reference's search loop (QuantizedGraph::
// search_qg_with_heap, symqglib/qg/qg.hpp:298-344) with both of its
// std::priority_queue pools emulated exactly in shared memory, one warp per
// query. It gives the reference's ids for every query, including those whose
// distances tie, where the binary-heap layout decides the order.
//
// Heaps: arrays of (id, distance bits) with comp(x, y) = x.dist < y.dist
// (qg.hpp:289-293); the search pool stores -distance. push and pop follow GCC
// libstdc++'s heap algorithms step for step:
//   push: append, then sift up while comp(parent, value). The path from the
//         new slot to the root is known in advance and comp(parent, value) is
//         monotone along it (a heap's values never decrease towards the root),
//         so lane i loads the i-th ancestor, one ballot gives how far the value
//         rises, and the shifted ancestors are written in one step.
//   pop:  move the last element out, walk a hole from the root to a leaf along
//         the larger child (the right one unless comp(right, left)), then sift
//         the moved element up from there. The walk is data dependent and runs
//         on lane 0; the sift-up is the warp-parallel one.
// Visited: the direct-mapped cache of the fast kernel (may forget, never
// invents). A forgotten node evaluated again has its old distance: it then
// fails the acceptance test (any trimmed or rejected node is at or above the
// current bound), or it is still in the result pool, which is checked before
// it could be pushed twice. So the accepted sequence equals the reference's.
// The search pool keeps its first scap slots in shared memory and the deeper
// heap levels in a per-warp global-memory area; a query whose search pool
// outgrows both goes to the global-memory exact kernel through a second list.
#include <cuda_runtime.h>
#include <math_constants.h>

#include "lqg_internal.h"
#include "lqg_kernels.cuh"
#include "heap_ops.cuh"
#include "sq8_batch.cuh"

namespace lqg {

using namespace heapops;

template <int G, int DEGW>
__global__ void __launch_bounds__(256, 2) heap_search_kernel(SearchArgs a, HeapArgs hp) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t dim = a.dim;
    const uint32_t dpad = (dim + 15u) & ~15u;
    float* pmin = reinterpret_cast<float*>(smem);
    float* pscale = pmin + dpad;
    const uint32_t vbits = a.vbits;
    const uint32_t vsize = 1u << vbits;
    unsigned char* wb = smem + 8u * dpad + (size_t)warp * heap_warp_bytes(dim, vbits, hp.rcap, hp.scap);
    float* qs = reinterpret_cast<float*>(wb);
    uint32_t* vis = reinterpret_cast<uint32_t*>(wb + 4u * dpad);
    uint32_t* cid = vis + vsize;
    float* cd = reinterpret_cast<float*>(cid + kMaxDeg);
    uint2* rps = reinterpret_cast<uint2*>(cd + kMaxDeg);
    const HeapView rp{rps, nullptr, hp.rcap};
    const size_t gw = (size_t)blockIdx.x * (blockDim.x >> 5) + warp;
    const HeapView sp{rps + hp.rcap, hp.sp_global + gw * hp.gcap, hp.scap};
    const uint32_t sp_max = hp.scap + hp.gcap;

    for (uint32_t i = threadIdx.x; i < dpad; i += blockDim.x) {
        pmin[i] = i < dim ? a.params[2 * i] : 0.f;
        pscale[i] = i < dim ? a.params[2 * i + 1] : 0.f;
    }
    __syncthreads();

    const int g = lane / G, r = lane % G;
    const uint32_t lt = lanemask_lt();
    const int64_t mlist = a.nlist ? (int64_t)*a.nlist : a.m;

    for (;;) {
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(a.qhead, 1u);
        slot = __shfl_sync(kFull, slot, 0);
        if ((int64_t)slot >= mlist) break;
        const int64_t qi = a.qlist ? (int64_t)a.qlist[slot] : (int64_t)slot;
        uint32_t ef = query_ef(a, qi);
        ef = min(max(ef, 1u), hp.rcap - 1u);
        const uint32_t k = min(a.kq ? a.kq[qi] : a.k0, a.kstride);
        const float* q = a.queries + (size_t)qi * dim;
        for (uint32_t i = lane; i < dpad; i += 32) qs[i] = i < dim ? q[i] : 0.f;
        for (uint32_t i = lane; i < vsize; i += 32) vis[i] = kNoId;
        __syncwarp();

        // qg.hpp:305-311
        const uint32_t ep = a.entry;
        if (lane == 0) cid[0] = ep;
        __syncwarp();
        eval_batch<G, G>(a, cid, cd, 0, 1, qs, pmin, pscale, g, r);
        __syncwarp();
        const float d0 = cd[0];
        uint32_t sn = 0, rn = 0;
        if (lane == 0) {
            sp.set(0, make_uint2(ep, __float_as_uint(-d0)));
            rp.set(0, make_uint2(ep, __float_as_uint(d0)));
            vis[hash_id(ep, vbits)] = ep;
        }
        sn = 1;
        rn = 1;
        float lower = d0;
        __syncwarp();
        uint32_t pops = 0, calcs = 1;
        bool overflow = false;

        for (;;) {
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

            // qg.hpp:329-335, in list order. The bound only falls within a
            // pop once the result pool is full, so a candidate that fails the
            // test at the start of the pop fails it later too.
            const bool full0 = rn >= ef;
            const float lower0 = lower;
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t c0 = w * 32;
                if (c0 >= ncand) break;
                const uint32_t c = c0 + lane;
                const bool pass = c < ncand && (!full0 || lower0 > cd[c]);
                unsigned pm = __ballot_sync(kFull, pass);
                while (pm) {
                    const int src = __ffs(pm) - 1;
                    pm &= pm - 1;
                    const uint32_t cc = c0 + src;
                    const float y = cd[cc];
                    const uint32_t id = cid[cc];
                    if (!(rn < ef || lower > y)) continue;
                    // a forgotten, already pooled node: the reference has it visited
                    bool in_rp = false;
                    for (uint32_t i = lane; i < rn; i += 32) in_rp |= rps[i].x == id;
                    if (__any_sync(kFull, in_rp)) continue;
                    if (sn + 1 > sp_max) {
                        overflow = true;
                        break;
                    }
                    warp_push(sp, sn, make_uint2(id, __float_as_uint(-y)), lane);
                    warp_push(rp, rn, make_uint2(id, __float_as_uint(y)), lane);
                    if (rn > ef) warp_pop(rp, rn, lane);
                    lower = __uint_as_float(rps[0].y);
                }
                if (overflow) break;
            }
            if (overflow) break;
        }

        if (overflow) {
            if (lane == 0) {
                const uint32_t i = atomicAdd(hp.nspill, 1u);
                hp.spill[i] = (int32_t)qi;
            }
            continue;
        }

        // qg.hpp:340-343
        const uint32_t P = rn;
        const uint32_t kk = min(k, P);
        uint32_t* out = a.ids + (size_t)qi * a.kstride;
        for (uint32_t j = lane; j < k - kk; j += 32) out[j] = kNoId;
        if (a.pool_ids)
            for (uint32_t j = P + lane; j < a.pstride; j += 32) {
                a.pool_ids[(size_t)qi * a.pstride + j] = kNoId;
                a.pool_d[(size_t)qi * a.pstride + j] = CUDART_INF_F;
            }
        // only the first k pops write ids; the rest matter for the pool output
        const uint32_t ex = a.pool_ids ? P : kk;
        for (uint32_t j = 0; j < ex; ++j) {
            const uint2 t = rps[0];
            if (lane == 0) {
                if (j < k) out[k - 1 - j] = t.x;
                const uint32_t pos = P - 1 - j;
                if (a.pool_ids && pos < a.pstride) {
                    a.pool_ids[(size_t)qi * a.pstride + pos] = t.x;
                    a.pool_d[(size_t)qi * a.pstride + pos] = __uint_as_float(t.y);
                }
            }
            warp_pop(rp, rn, lane);
        }
        if (a.stats && lane == 0) {
            uint4 st = make_uint4(pops, calcs, 1u, P);
            *reinterpret_cast<uint4*>(a.stats + 4 * (size_t)qi) = st;
        }
        __syncwarp();
    }
}

size_t heap_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t rcap, uint32_t scap, int warps) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 8 * dpad + (size_t)warps * heap_warp_bytes(dim, vbits, rcap, scap);
}

template <int G, int DEGW>
static cudaError_t heap_run(const SearchArgs& a, const HeapArgs& h, int warps, int blocks,
                            cudaStream_t st, int* occ) {
    const size_t smem = heap_smem_bytes(a.dim, a.vbits, h.rcap, h.scap, warps);
    auto k = heap_search_kernel<G, DEGW>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, warps * 32, smem);
    k<<<blocks, warps * 32, smem, st>>>(a, h);
    return cudaGetLastError();
}

cudaError_t launch_heap(const SearchArgs& a, const HeapArgs& h, int G, int degw, int warps,
                        int blocks, cudaStream_t st, int* occ) {
#define LQG_HCASE(GG, DW) \
    if (G == GG && degw == DW) return heap_run<GG, DW>(a, h, warps, blocks, st, occ);
#define LQG_HCASES(GG) LQG_HCASE(GG, 1) LQG_HCASE(GG, 2) LQG_HCASE(GG, 3) LQG_HCASE(GG, 4)
    LQG_HCASES(1)
    LQG_HCASES(2)
    LQG_HCASES(4)
    LQG_HCASES(8)
    LQG_HCASES(16)
#undef LQG_HCASES
#undef LQG_HCASE
    return cudaErrorInvalidValue;
}

}  // namespace lqg
