// Device side of the B200 quantized-graph query path: shared helpers.
//
// Distance arithmetic restates, bit for bit, what one neighbour evaluation of
// the reference computes (symqglib/qg/qg.hpp:325-328):
//   dec[d]  = fma(code[d], scale[d], min[d])   (sq8.hpp:28-32, contracted by -Ofast)
//   t       = q[d] - dec[d]
//   acc[l]  = fma(t, t, acc[l]),  l = d % 16, in increasing d  (l2.hpp:16-35)
//   result  = _mm512_reduce_add_ps tree: fold lanes 8..15 onto 0..7, then
//             4..7 onto 0..3, 2..3 onto 0..1, 1 onto 0; then a scalar fma
//             tail over d >= 16*floor(D/16).
// A warp evaluates 32/G candidates at once: the G lanes of a group each own
// 16/G of the 16 accumulators, and the fold tree runs across them with
// shuffles. All arithmetic uses the _rn intrinsics, which the compiler never
// fuses or reorders.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lqg {

constexpr uint32_t kExpanded = 0x80000000u;  // pool id flag: node already popped
constexpr uint32_t kNoId = 0xFFFFFFFFu;
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint32_t kMaxDeg = 128;                 // degree_bound 32, 64, 96 or 128
constexpr uint32_t kCandBytes = 8 * kMaxDeg;      // per-warp candidate staging

struct SearchArgs {
    const uint32_t* nbrs;    // [n][deg]
    const uint8_t* codes;    // [n][cstride]
    const float* params;     // [dim][2] (min, scale)
    uint32_t n, dim, deg, cstride, entry;
    const float* queries;    // [m][dim]
    int64_t m;               // number of queries in the work list
    const int32_t* qlist;    // work list of query indices (NULL: 0..m-1)
    const uint32_t* nlist;   // if set, the work list length is *nlist (<= m)
    const uint32_t* kq;      // per-query k or NULL
    uint32_t k0;
    const uint32_t* efq;     // per-query ef or NULL
    uint32_t ef0;
    uint32_t* ids;           // [.][kstride]
    uint32_t kstride;
    uint32_t* pool_ids;      // [.][pstride] or NULL
    float* pool_d;
    uint32_t pstride;
    uint32_t* stats;         // [.][4] or NULL
    int32_t* flagged;        // fast kernel: queries handed to the exact kernel
    uint32_t* nflagged;
    uint32_t* qhead;         // work-queue head (zeroed before each launch)
    uint32_t* err;           // [0]: error bits, [1]: first failing query
    uint32_t vbits;          // fast kernel: visited-cache bits
    uint32_t ties_ok;        // fast kernel: resolve equal distances by insertion
                             // order instead of handing the query to the exact
                             // kernel (index build only; not reference order)
    uint32_t* path;          // fast kernel (index build): the first path_stride
    uint32_t path_stride;    // popped ids of each query, padded with kNoId
};

// Exact kernel work areas, one per resident warp.
struct ExactScratch {
    uint32_t* vis;     // [warps][1 << xbits] exact visited hash set
    uint2* sp;         // [warps][scap]  (id, -dist bits) heap
    uint2* rp;         // [warps][rcap]  (id, dist bits) heap
    uint32_t xbits;
    uint32_t scap;
    uint32_t rcap;
};

enum : uint32_t {
    kErrVisitedFull = 1u,
    kErrHeapFull = 2u,
    kErrProbe = 4u,
    kErrSync = 8u,  // replay kernel: a bounded wait between its warps ran out
};

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ef of query qi: its per-query value when the caller gave an array, clamped
// to [1, ef0] (ef0 is the batch's bound, checked on the host to be <= 512), so
// a per-query value above the bound runs at the bound.
__device__ __forceinline__ uint32_t query_ef(const SearchArgs& a, int64_t qi) {
    const uint32_t e = a.efq ? a.efq[qi] : a.ef0;
    return min(max(e, 1u), max(a.ef0, 1u));
}

__device__ __forceinline__ uint32_t hash_id(uint32_t v, uint32_t bits) {
    return (v * 0x9E3779B1u) >> (32u - bits);
}

// byte t of w as an exact float: 0x4B0000bb is 2^23 + bb.
__device__ __forceinline__ float byte_to_float(uint32_t w, int t) {
    return __fsub_rn(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u + t)), 8388608.0f);
}

// Loads the A = 16/G code bytes of chunk j owned by lane r of a group into w[].
template <int A>
__device__ __forceinline__ void load_chunk(const uint8_t* p, uint32_t (&w)[(A + 3) / 4]) {
    if constexpr (A == 16) {
        uint4 x = __ldg(reinterpret_cast<const uint4*>(p));
        w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
    } else if constexpr (A == 8) {
        uint2 x = __ldg(reinterpret_cast<const uint2*>(p));
        w[0] = x.x; w[1] = x.y;
    } else if constexpr (A == 4) {
        w[0] = __ldg(reinterpret_cast<const uint32_t*>(p));
    } else if constexpr (A == 2) {
        w[0] = __ldg(reinterpret_cast<const unsigned short*>(p));
    } else {
        w[0] = __ldg(p);
    }
}

// A consecutive floats from shared memory (16-byte aligned when A >= 4).
template <int A>
__device__ __forceinline__ void load_vec(const float* p, float (&v)[A]) {
    if constexpr (A >= 4) {
#pragma unroll
        for (int i = 0; i < A / 4; ++i) {
            float4 x = reinterpret_cast<const float4*>(p)[i];
            v[4 * i] = x.x; v[4 * i + 1] = x.y; v[4 * i + 2] = x.z; v[4 * i + 3] = x.w;
        }
    } else if constexpr (A == 2) {
        float2 x = *reinterpret_cast<const float2*>(p);
        v[0] = x.x; v[1] = x.y;
    } else {
        v[0] = p[0];
    }
}

// ---- packed FP32 pairs -----------------------------------------------------

__device__ __forceinline__ unsigned long long pk(uint32_t lo, uint32_t hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(lo), "r"(hi));
    return r;
}
__device__ __forceinline__ void upk(unsigned long long v, float& lo, float& hi) {
    uint32_t a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=r"(a), "=r"(b) : "l"(v));
    lo = __uint_as_float(a);
    hi = __uint_as_float(b);
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Squared L2 between the query (shared memory, qs) and the SQ8-decoded row.
// Called by all 32 lanes together; lane r = lane % G of each group handles
// accumulators [r*A, r*A + A). `valid` lanes load; the others compute on
// zeros. The result is meaningful in lane r == 0 of each group.
template <int G>
__device__ __forceinline__ float sq8_l2_group(const uint8_t* row, bool valid,
                                              const float* __restrict__ qs,
                                              const float* __restrict__ pmin,
                                              const float* __restrict__ pscale,
                                              uint32_t dim, int r) {
    constexpr int A = 16 / G;
    constexpr int W = (A + 3) / 4;
    float acc[A];
#pragma unroll
    for (int t = 0; t < A; ++t) acc[t] = 0.0f;
    const uint32_t mul = dim & ~15u;
    const uint8_t* p = row + r * A;
    // Up to U chunks of the row are requested before any arithmetic, so the
    // global-memory latency is paid once per U chunks, not once per chunk.
    constexpr int U = 8;
    // A >= 2: the arithmetic on packed FP32 pairs (fma.rn.f32x2 and
    // sub.rn.f32x2 round each half exactly as the scalar instructions do)
    constexpr int AP = A >= 2 ? A / 2 : 1;
    unsigned long long acc2[AP];
#pragma unroll
    for (int t = 0; t < AP; ++t) acc2[t] = 0ull;
    const unsigned long long C23 = pk(0x4B000000u, 0x4B000000u);
    for (uint32_t base = 0; base < mul; base += 16 * U) {
        uint32_t w[U][W];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t b = base + 16 * u;
            if (valid && b < mul) {
                load_chunk<A>(p + b, w[u]);
            } else {
#pragma unroll
                for (int i = 0; i < W; ++i) w[u][i] = 0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t d0 = base + 16 * u + r * A;
            if (base + 16 * u < mul) {
                if constexpr (A >= 2) {
                    unsigned long long q2[AP], m2[AP], s2[AP];
                    if constexpr (AP >= 2) {
#pragma unroll
                        for (int t = 0; t < AP; t += 2) {
                            const ulonglong2 qq = *reinterpret_cast<const ulonglong2*>(qs + d0 + 2 * t);
                            const ulonglong2 mm = *reinterpret_cast<const ulonglong2*>(pmin + d0 + 2 * t);
                            const ulonglong2 ss = *reinterpret_cast<const ulonglong2*>(pscale + d0 + 2 * t);
                            q2[t] = qq.x;
                            q2[t + 1] = qq.y;
                            m2[t] = mm.x;
                            m2[t + 1] = mm.y;
                            s2[t] = ss.x;
                            s2[t + 1] = ss.y;
                        }
                    } else {
                        q2[0] = *reinterpret_cast<const unsigned long long*>(qs + d0);
                        m2[0] = *reinterpret_cast<const unsigned long long*>(pmin + d0);
                        s2[0] = *reinterpret_cast<const unsigned long long*>(pscale + d0);
                    }
#pragma unroll
                    for (int t = 0; t < AP; ++t) {
                        const uint32_t wd = w[u][(2 * t) / 4];
                        const int s0 = (2 * t) % 4;
                        const uint32_t lo = __byte_perm(wd, 0x4B000000u, 0x7440u + s0);
                        const uint32_t hi = __byte_perm(wd, 0x4B000000u, 0x7440u + s0 + 1);
                        const unsigned long long c2 = sub2(pk(lo, hi), C23);
                        const unsigned long long dec = fma2(c2, s2[t], m2[t]);
                        const unsigned long long df = sub2(q2[t], dec);
                        acc2[t] = fma2(df, df, acc2[t]);
                    }
                } else {
                    float qv[A], mv[A], sv[A];
                    load_vec<A>(qs + d0, qv);
                    load_vec<A>(pmin + d0, mv);
                    load_vec<A>(pscale + d0, sv);
#pragma unroll
                    for (int t = 0; t < A; ++t) {
                        float c = byte_to_float(w[u][t / 4], t % 4);
                        float dec = __fmaf_rn(c, sv[t], mv[t]);
                        float df = __fsub_rn(qv[t], dec);
                        acc[t] = __fmaf_rn(df, df, acc[t]);
                    }
                }
            }
        }
    }
    if constexpr (A >= 2) {
#pragma unroll
        for (int t = 0; t < AP; ++t) upk(acc2[t], acc[2 * t], acc[2 * t + 1]);
    }
    // fold tree: h = 8, 4, 2, 1
#pragma unroll
    for (int h = 8; h >= 1; h >>= 1) {
        if (h >= A) {
#pragma unroll
            for (int t = 0; t < A; ++t) {
                float o = __shfl_down_sync(kFull, acc[t], h / A);
                acc[t] = __fadd_rn(acc[t], o);
            }
        } else {
#pragma unroll
            for (int t = 0; t < A; ++t)
                if (t < h) acc[t] = __fadd_rn(acc[t], acc[t + h]);
        }
    }
    float res = acc[0];
    if (mul < dim && r == 0 && valid) {
        for (uint32_t d = mul; d < dim; ++d) {
            float c = (float)row[d];
            float dec = __fmaf_rn(c, pscale[d], pmin[d]);
            float df = __fsub_rn(qs[d], dec);
            res = __fmaf_rn(df, df, res);
        }
    }
    return res;
}

}  // namespace lqg
