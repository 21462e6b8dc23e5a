// Exact search kernel (libstdc++ heap emulation) and its launcher.
#include <cuda_runtime.h>
#include <math_constants.h>

#include "lqg_internal.h"
#include "lqg_kernels.cuh"

namespace lqg {

// ---- exact kernel --------------------------------------------------------

// GCC libstdc++ heap steps on (id, distance-bits) pairs; comp(x, y) is
// x.dist < y.dist (symqglib/qg/qg.hpp:289-293).
__device__ __forceinline__ bool hcomp(uint2 x, uint2 y) {
    return __uint_as_float(x.y) < __uint_as_float(y.y);
}

__device__ void heap_sift_up(uint2* h, uint32_t hole, uint32_t top, uint2 v) {
    uint32_t parent = (hole - 1) / 2;
    while (hole > top && hcomp(h[parent], v)) {
        h[hole] = h[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    h[hole] = v;
}

__device__ void heap_push(uint2* h, uint32_t& n, uint2 v) {
    h[n] = v;
    heap_sift_up(h, n, 0, v);
    ++n;
}

__device__ void heap_pop(uint2* h, uint32_t& n) {
    const uint32_t size = n;
    if (size > 1) {
        const uint32_t len = size - 1;
        const uint2 v = h[len];
        h[len] = h[0];
        uint32_t hole = 0, second = 0;
        while (second < (len - 1) / 2) {
            second = 2 * (second + 1);
            if (hcomp(h[second], h[second - 1])) second--;
            h[hole] = h[second];
            hole = second;
        }
        if ((len & 1u) == 0 && second == (len - 2) / 2) {
            second = 2 * (second + 1);
            h[hole] = h[second - 1];
            hole = second - 1;
        }
        heap_sift_up(h, hole, 0, v);
    }
    n = size - 1;
}

// Exact set insert; true if v was absent. Open addressing, linear probing.
__device__ __forceinline__ bool vis_insert(uint32_t* vis, uint32_t v, uint32_t bits,
                                           bool& fail) {
    const uint32_t mask = (1u << bits) - 1u;
    uint32_t h = hash_id(v, bits);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        const uint32_t prev = atomicCAS(vis + h, kNoId, v);
        if (prev == kNoId) return true;
        if (prev == v) return false;
        h = (h + 1u) & mask;
    }
    fail = true;
    return false;
}

template <int G, int DEGW>
__global__ void __launch_bounds__(256) exact_search_kernel(SearchArgs a, ExactScratch s) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const uint32_t dim = a.dim;
    const uint32_t dpad = (dim + 15u) & ~15u;
    float* pmin = reinterpret_cast<float*>(smem);
    float* pscale = pmin + dpad;
    unsigned char* wb = smem + 8u * dpad + (size_t)warp * (4u * dpad + kCandBytes);
    float* qs = reinterpret_cast<float*>(wb);
    uint32_t* cid = reinterpret_cast<uint32_t*>(wb + 4u * dpad);
    float* cd = reinterpret_cast<float*>(cid + kMaxDeg);

    for (uint32_t i = threadIdx.x; i < dpad; i += blockDim.x) {
        pmin[i] = i < dim ? a.params[2 * i] : 0.f;
        pscale[i] = i < dim ? a.params[2 * i + 1] : 0.f;
    }
    __syncthreads();

    const size_t gw = (size_t)blockIdx.x * nwarps + warp;
    uint32_t* vis = s.vis + (gw << s.xbits);
    uint2* sp = s.sp + gw * s.scap;
    uint2* rp = s.rp + gw * s.rcap;
    const uint32_t vsize = 1u << s.xbits;
    const uint32_t vlimit = vsize >> 1;
    const int g = lane / G, r = lane % G;
    constexpr int CPP = 32 / G;
    const uint32_t lt = lanemask_lt();
    const int64_t mlist = a.nlist ? (int64_t)*a.nlist : a.m;

    for (;;) {
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(a.qhead, 1u);
        slot = __shfl_sync(kFull, slot, 0);
        if ((int64_t)slot >= mlist) break;
        const int64_t qi = a.qlist ? (int64_t)a.qlist[slot] : (int64_t)slot;
        uint32_t ef = query_ef(a, qi);
        ef = min(max(ef, 1u), s.rcap - 1u);
        const uint32_t k = min(a.kq ? a.kq[qi] : a.k0, a.kstride);
        const float* q = a.queries + (size_t)qi * dim;
        for (uint32_t i = lane; i < dpad; i += 32) qs[i] = i < dim ? q[i] : 0.f;
        for (uint32_t i = lane; i < vsize; i += 32) vis[i] = kNoId;
        __syncwarp();

        bool fail = false;
        uint32_t failbits = 0;
        const uint32_t ep = a.entry;
        float d0 = sq8_l2_group<G>(a.codes + (size_t)ep * a.cstride, g == 0, qs, pmin,
                                   pscale, dim, r);
        d0 = __shfl_sync(kFull, d0, 0);
        uint32_t sn = 0, rn = 0;  // heap sizes (lane 0)
        float lower = d0;
        if (lane == 0) {
            heap_push(sp, sn, make_uint2(ep, __float_as_uint(-d0)));
            heap_push(rp, rn, make_uint2(ep, __float_as_uint(d0)));
            vis_insert(vis, ep, s.xbits, fail);
        }
        __syncwarp();
        uint32_t pops = 0, evals = 0, nvis = 1;

        for (;;) {
            int go = 0;
            uint32_t u = 0;
            if (lane == 0 && sn > 0) {
                const uint2 top = sp[0];
                if (!(-__uint_as_float(top.y) > lower)) {
                    go = 1;
                    u = top.x;
                    heap_pop(sp, sn);
                }
            }
            go = __shfl_sync(kFull, go, 0);
            if (!go) break;
            u = __shfl_sync(kFull, u, 0);
            ++pops;

            uint32_t ncand = 0;
            const uint32_t* nb = a.nbrs + (size_t)u * a.deg;
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t v = __ldg(nb + w * 32 + lane);
                const unsigned mm = __match_any_sync(kFull, v);
                bool fresh = false;
                if ((mm & lt) == 0) fresh = vis_insert(vis, v, s.xbits, fail);
                const unsigned kb = __ballot_sync(kFull, fresh);
                if (fresh) cid[ncand + __popc(kb & lt)] = v;
                ncand += __popc(kb);
                __syncwarp();
            }
            nvis += ncand;
            if (nvis > vlimit) {
                fail = true;
                failbits |= kErrVisitedFull;
            }
            for (uint32_t base = 0; base < ncand; base += CPP) {
                const uint32_t c = base + g;
                const bool valid = c < ncand;
                const uint32_t id = valid ? cid[c] : 0u;
                const float d = sq8_l2_group<G>(a.codes + (size_t)id * a.cstride, valid, qs,
                                                pmin, pscale, dim, r);
                if (valid && r == 0) cd[c] = d;
            }
            evals += ncand;
            __syncwarp();
            if (lane == 0) {
                for (uint32_t c = 0; c < ncand && !fail; ++c) {
                    const float y = cd[c];
                    if (rn < ef || lower > y) {
                        if (sn + 1 >= s.scap) {
                            fail = true;
                            failbits |= kErrHeapFull;
                            break;
                        }
                        heap_push(sp, sn, make_uint2(cid[c], __float_as_uint(-y)));
                        heap_push(rp, rn, make_uint2(cid[c], __float_as_uint(y)));
                        if (rn > ef) heap_pop(rp, rn);
                        lower = __uint_as_float(rp[0].y);
                    }
                }
            }
            lower = __shfl_sync(kFull, lower, 0);
            fail = __any_sync(kFull, fail);
            __syncwarp();
            if (fail) break;
        }

        uint32_t* out = a.ids + (size_t)qi * a.kstride;
        if (__any_sync(kFull, fail)) {
            failbits = __reduce_or_sync(kFull, failbits);
            if (!failbits) failbits = kErrProbe;
            for (uint32_t j = lane; j < k; j += 32) out[j] = kNoId;
            if (lane == 0) {
                atomicOr(a.err, failbits);
                atomicCAS(a.err + 1, kNoId, (uint32_t)qi);
            }
            continue;
        }
        const uint32_t P = __shfl_sync(kFull, rn, 0);
        const uint32_t kk = min(k, P);
        for (uint32_t j = lane; j < k - kk; j += 32) out[j] = kNoId;
        if (a.pool_ids)
            for (uint32_t j = P + lane; j < a.pstride; j += 32) {
                a.pool_ids[(size_t)qi * a.pstride + j] = kNoId;
                a.pool_d[(size_t)qi * a.pstride + j] = CUDART_INF_F;
            }
        if (lane == 0) {
            for (uint32_t j = 0; rn > 0; ++j) {
                const uint2 t = rp[0];
                if (j < k) out[k - 1 - j] = t.x;
                const uint32_t pos = P - 1 - j;
                if (a.pool_ids && pos < a.pstride) {
                    a.pool_ids[(size_t)qi * a.pstride + pos] = t.x;
                    a.pool_d[(size_t)qi * a.pstride + pos] = __uint_as_float(t.y);
                }
                heap_pop(rp, rn);
            }
            if (a.stats) {
                uint4 st = make_uint4(pops, evals, 2u, P);
                *reinterpret_cast<uint4*>(a.stats + 4 * (size_t)qi) = st;
            }
        }
        __syncwarp();
    }
}

size_t exact_smem_bytes(uint32_t dim, int warps) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 8 * dpad + (size_t)warps * (4 * dpad + kCandBytes);
}

template <int G, int DEGW>
static cudaError_t run_exact(const SearchArgs& a, const ExactScratch& s, int warps,
                             int blocks, cudaStream_t st) {
    const size_t smem = exact_smem_bytes(a.dim, warps);
    auto k = exact_search_kernel<G, DEGW>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k<<<blocks, warps * 32, smem, st>>>(a, s);
    return cudaGetLastError();
}

cudaError_t launch_exact(const SearchArgs& a, const ExactScratch& s, int degw, int warps,
                         int blocks, cudaStream_t st) {
    // The exact kernel's time goes to its serial heap work; 4 lanes per
    // candidate is a fixed, adequate split of the distance work.
    switch (degw) {
        case 1: return run_exact<4, 1>(a, s, warps, blocks, st);
        case 2: return run_exact<4, 2>(a, s, warps, blocks, st);
        case 3: return run_exact<4, 3>(a, s, warps, blocks, st);
        case 4: return run_exact<4, 4>(a, s, warps, blocks, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lqg
