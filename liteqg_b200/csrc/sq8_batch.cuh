// Batched SQ8 decode + squared L2 of up to 32 candidates per call, shared by
// the heap and replay search kernels. Bit-exact with the reference's
// evaluation (symqglib/qg/qg.hpp:325-328): decode fma(code, scale, min)
// (sq8.hpp:28-32, contracted by -Ofast), then 16 accumulators
// acc[d % 16] = fma(q - dec, q - dec, acc) in increasing d and the AVX-512
// reduction tree (l2.hpp:16-35), then the scalar tail for D % 16.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lqg_kernels.cuh"

namespace lqg {

// Rows of at least this many code bytes ("wide") need a longer code-load
// window than narrow ones: the window is counted in 16-byte chunks per round.
constexpr uint32_t kBatchWideDim = 256;

// Distances of candidates cid[base + p * (32/G) + g], p < NP, into cd[].
// Lane r of group g owns accumulators [r*A, r*A + A) (A = 16/G); all code
// bytes of a round of U chunks, for all NP passes, are requested before any
// arithmetic: LW code words per lane in flight (U = LW / (NP * words per
// chunk), at most 8). With PF, each round first asks L1 for the next round's
// bytes of every row, so a row split over two rounds costs one trip to L2 or
// HBM. Passes with no valid candidate are skipped (warp-uniform).
template <int G, int NP, int LW = 32, int PF = 0>
__device__ __forceinline__ void eval_batch(const SearchArgs& a, const uint32_t* cid, float* cd,
                                           uint32_t base, uint32_t ncand,
                                           const float* __restrict__ qs,
                                           const float* __restrict__ pmin,
                                           const float* __restrict__ pscale, int g, int r) {
    constexpr int A = 16 / G;
    constexpr int W = (A + 3) / 4;
    constexpr int CPP = 32 / G;
    constexpr int UU = LW / (NP * W);
    constexpr int U = UU < 1 ? 1 : (UU > 8 ? 8 : UU);
    constexpr int AP = A >= 2 ? A / 2 : 1;  // accumulator pairs
    const uint32_t dim = a.dim;
    const uint32_t mul = dim & ~15u;
    const unsigned long long C23 = pk(0x4B000000u, 0x4B000000u);

    const uint8_t* rowp[NP];
    bool valid[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const uint32_t c = base + p * CPP + g;
        valid[p] = c < ncand;
        rowp[p] = a.codes + (size_t)(valid[p] ? cid[c] : 0u) * a.cstride + r * A;
    }
    unsigned long long acc2[NP][AP];
    float acc1[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        acc1[p] = 0.f;
#pragma unroll
        for (int t = 0; t < AP; ++t) acc2[p][t] = 0ull;
    }
    for (uint32_t b0 = 0; b0 < mul; b0 += 16 * U) {
        if constexpr (PF != 0) {
#pragma unroll
            for (int p = 0; p < NP; ++p)
                if (valid[p] && b0 + 16 * U < mul)
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(rowp[p] + b0 + 16 * U));
        }
        uint32_t w[NP][U][W];
#pragma unroll
        for (int p = 0; p < NP; ++p)
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t b = b0 + 16 * u;
                if (valid[p] && b < mul) {
                    load_chunk<A>(rowp[p] + b, w[p][u]);
                } else {
#pragma unroll
                    for (int i = 0; i < W; ++i) w[p][u][i] = 0;
                }
            }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t b = b0 + 16 * u;
            if (b >= mul) break;
            const uint32_t d0 = b + r * A;
            if constexpr (A >= 2) {
                // query, min and scale pairs: 16-byte loads where a lane owns
                // 4 or more dimensions of the chunk (every caller's arrays
                // start on 16 bytes, and d0 is a multiple of A)
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
                for (int p = 0; p < NP; ++p) {
                    if (base + p * CPP >= ncand) continue;
#pragma unroll
                    for (int t = 0; t < AP; ++t) {
                        const uint32_t wd = w[p][u][(2 * t) / 4];
                        const int s0 = (2 * t) % 4;
                        const uint32_t lo = __byte_perm(wd, 0x4B000000u, 0x7440u + s0);
                        const uint32_t hi = __byte_perm(wd, 0x4B000000u, 0x7440u + s0 + 1);
                        const unsigned long long c2 = sub2(pk(lo, hi), C23);
                        const unsigned long long dec = fma2(c2, s2[t], m2[t]);
                        const unsigned long long df = sub2(q2[t], dec);
                        acc2[p][t] = fma2(df, df, acc2[p][t]);
                    }
                }
            } else {
                const float qv = qs[d0], mv = pmin[d0], sv = pscale[d0];
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    if (base + p * CPP >= ncand) continue;
                    const float c = byte_to_float(w[p][u][0], 0);
                    const float dec = __fmaf_rn(c, sv, mv);
                    const float df = __fsub_rn(qv, dec);
                    acc1[p] = __fmaf_rn(df, df, acc1[p]);
                }
            }
        }
    }
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        if (base + p * CPP >= ncand) break;  // warp-uniform
        float acc[A];
        if constexpr (A >= 2) {
#pragma unroll
            for (int t = 0; t < AP; ++t) upk(acc2[p][t], acc[2 * t], acc[2 * t + 1]);
        } else {
            acc[0] = acc1[p];
        }
        // the AVX-512 reduction tree (l2.hpp:16-35): fold 8, 4, 2, 1
#pragma unroll
        for (int h = 8; h >= 1; h >>= 1) {
            if (h >= A) {
#pragma unroll
                for (int t = 0; t < A; ++t) {
                    const float o = __shfl_down_sync(kFull, acc[t], h / A);
                    acc[t] = __fadd_rn(acc[t], o);
                }
            } else {
#pragma unroll
                for (int t = 0; t < A; ++t)
                    if (t < h) acc[t] = __fadd_rn(acc[t], acc[t + h]);
            }
        }
        float res = acc[0];
        const uint32_t c = base + p * CPP + g;
        if (r == 0 && valid[p]) {
            const uint8_t* row = a.codes + (size_t)cid[c] * a.cstride;
            for (uint32_t d = mul; d < dim; ++d) {
                const float cv = (float)row[d];
                const float dec = __fmaf_rn(cv, pscale[d], pmin[d]);
                const float df = __fsub_rn(qs[d], dec);
                res = __fmaf_rn(df, df, res);
            }
            cd[c] = res;
        }
    }
}

}  // namespace lqg
