/* Test infrastructure only (see fs_oracle.h): the CPU oracle for the upstream
 * FastScan/RaBitQ query path. Each function cites the reference code it
 * restates (paths relative to the LiteQG project root). Compiled without
 * fast-math and without FP contraction: every fused multiply-add is an
 * explicit fmaf(), as the reference's -Ofast AVX-512 build emits it. */
#include "fs_oracle.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

uint32_t fso_padded_dim(uint32_t dim) {
    uint32_t p = 1;
    while (p < dim) p <<= 1;
    return p;
}

/* The FFHT kernels the reference's rotator calls (third/ffht, helper_float_N)
 * run log2(P) butterfly stages, (a, b) -> (a + b, a - b) on the pairs that
 * differ in one index bit, from the lowest bit to the highest. */
void fso_fht(float* buf, uint32_t logp) {
    const uint32_t n = 1u << logp;
    for (uint32_t h = 1; h < n; h <<= 1)
        for (uint32_t i = 0; i < n; i += 2 * h)
            for (uint32_t j = i; j < i + h; ++j) {
                const float a = buf[j], b = buf[j + h];
                buf[j] = a + b;
                buf[j + h] = a - b;
            }
}

/* utils/rotator.hpp:89-114: element-wise product with the diagonal, zero
 * padding to P, then the transform (the diagonal carries the 1/sqrt(P)). */
void fso_rotate(const float* src, uint32_t dim, uint32_t P, const float* diag, float* dst) {
    uint32_t logp = 0;
    while ((1u << logp) < P) ++logp;
    for (uint32_t i = 0; i < dim; ++i) dst[i] = src[i] * diag[i];
    for (uint32_t i = dim; i < P; ++i) dst[i] = 0.0f;
    fso_fht(dst, logp);
}

/* qg/qg_query.hpp:30-45 with utils/scalar_quantize.hpp:12-58 and
 * quantization/fastscan_impl.hpp:258-270.
 * data_range, AVX-512 branch: the vector min/max start from zero, so
 * lower <= 0 <= upper. width = (upper - lower) / 63 (QG_BQUERY = 6,
 * common.hpp:11); the reference's -Ofast build evaluates it as
 * (upper - lower) * fl(1/63), and, having inlined quantize(), folds its
 * 1 / width into fl(1 / fl(1/63)) / (upper - lower) (= 62.999996f / range),
 * as its compiled code shows. Each value becomes round((v - lower) * that +
 * 0.5), the + 0.5 in double precision and the rounding half away from zero
 * (std::lround, which the build expands as trunc(x + 0.49999999999999994) for
 * x > 0); sumq is their sum. The lookup table of
 * 4-dimension group g holds, for each nibble j, the sum of the group's
 * quantized values whose bit is set in j, the group's first dimension on
 * bit 3 (kPos), in 8-bit arithmetic. */
void fso_query_prepare(const float* rot, uint32_t P, uint8_t* lut, float* width, float* lower,
                       int32_t* sumq) {
    float lo = 0.0f, hi = 0.0f;
    for (uint32_t i = 0; i < P; ++i) {
        lo = rot[i] < lo ? rot[i] : lo;
        hi = rot[i] > hi ? rot[i] : hi;
    }
    const float range = hi - lo;
    const float w = range * (1.0f / 63.0f);
    const float inv = (1.0f / (1.0f / 63.0f)) / range;
    uint8_t* bq = (uint8_t*)malloc(P);
    int32_t s = 0;
    for (uint32_t i = 0; i < P; ++i) {
        const float t = (rot[i] - lo) * inv;
        bq[i] = (uint8_t)trunc(((double)t + 0.5) + 0.49999999999999994);
        s += bq[i];
    }
    for (uint32_t g = 0; g < P / 4; ++g) {
        uint8_t* L = lut + 16 * g;
        for (int j = 0; j < 16; ++j) {
            uint8_t v = 0;
            for (int b = 0; b < 4; ++b)
                if (j & (1 << b)) v = (uint8_t)(v + bq[4 * g + 3 - b]);
            L[j] = v;
        }
    }
    free(bq);
    *width = w;
    *lower = lo;
    *sumq = s;
}

/* quantization/rabitq.hpp:23-108: residual r = rot_nb - rot_c; sign bits
 * r > 0; x = |r|, x0 = <r, sign(r)> / (sqrt(P) x), x1 = <rot_c, sign(r)> / sqrt(P);
 *   triple_x  = x^2 + 2 (x / x0) x1
 *   factor_dq = -2 (x / x0) / sqrt(P)
 *   factor_vq = -2 (x / x0) / sqrt(P) * (2 popcount - P) */
void fso_rabitq(const float* rot_nb, const float* rot_c, uint32_t deg, uint32_t P,
                uint8_t* bits, float* factors) {
    const double fac_norm = 1.0 / sqrt((double)P);
    for (uint32_t j = 0; j < deg; ++j) {
        const float* o = rot_nb + (size_t)j * P;
        uint8_t* bj = bits + (size_t)j * (P / 8);
        memset(bj, 0, P / 8);
        double nrm2 = 0.0, dotx = 0.0, dotc = 0.0;
        int pop = 0;
        for (uint32_t d = 0; d < P; ++d) {
            const float r = o[d] - rot_c[d];
            const int s = r > 0.0f;
            const double sg = s ? 1.0 : -1.0;
            nrm2 += (double)r * (double)r;
            dotx += (double)r * sg;
            dotc += (double)rot_c[d] * sg;
            pop += s;
            if (s) {
                const uint32_t byte = d / 8, t = d % 8;
                bj[byte] |= (uint8_t)(t < 4 ? (1u << (3 - t)) : (1u << (7 - (t - 4))));
            }
        }
        const double x = sqrt(nrm2);
        if (!(x > 0.0)) {
            factors[j] = 0.0f;
            factors[deg + j] = 0.0f;
            factors[2 * deg + j] = 0.0f;
            continue;
        }
        const double x0 = dotx * fac_norm / x;
        const double x1 = dotc * fac_norm;
        const double xx0 = x / x0;
        factors[j] = (float)(x * x + 2.0 * xx0 * x1);
        factors[deg + j] = (float)(-2.0 * xx0 * fac_norm);
        factors[2 * deg + j] = (float)(-2.0 * xx0 * fac_norm * (double)(2 * pop - (int)P));
    }
}

/* quantization/fastscan_impl.hpp:43 (kPerm0), 63-95 (pack_codes_helper). */
static const int kPerm0[16] = {0, 8, 1, 9, 2, 10, 3, 11, 4, 12, 5, 13, 6, 14, 7, 15};

void fso_pack_codes(const uint8_t* bits, uint32_t ncode, uint32_t P, uint8_t* packed) {
    const uint32_t ncb = P / 4, rowb = P / 8;
    uint8_t* out = packed;
    for (uint32_t blk = 0; blk < ncode; blk += 32)
        for (uint32_t i = 0; i < ncb; i += 2) {
            uint8_t lo[32], hi[32];
            for (int j = 0; j < 32; ++j) {
                const uint8_t c = bits[(size_t)(blk + j) * rowb + i / 2];
                lo[j] = c & 15;
                hi[j] = c >> 4;
            }
            for (int j = 0; j < 16; ++j) {
                out[j] = (uint8_t)(lo[kPerm0[j]] | (lo[kPerm0[j] + 16] << 4));
                out[j + 16] = (uint8_t)(hi[kPerm0[j]] | (hi[kPerm0[j] + 16] << 4));
            }
            out += 32;
        }
}

void fso_unpack_codes(const uint8_t* packed, uint32_t ncode, uint32_t P, uint8_t* bits) {
    const uint32_t ncb = P / 4, rowb = P / 8;
    const uint8_t* in = packed;
    for (uint32_t blk = 0; blk < ncode; blk += 32)
        for (uint32_t i = 0; i < ncb; i += 2) {
            for (int j = 0; j < 16; ++j) {
                const int v = kPerm0[j];
                const uint8_t a = in[j], b = in[j + 16];
                /* vector v: codebook i in a's low nibble, i+1 in b's low nibble;
                   vector v+16: the high nibbles */
                bits[(size_t)(blk + v) * rowb + i / 2] = (uint8_t)((a & 15) | ((b & 15) << 4));
                bits[(size_t)(blk + v + 16) * rowb + i / 2] = (uint8_t)((a >> 4) | ((b >> 4) << 4));
            }
            in += 32;
        }
}

/* fastscan_impl.hpp:127-255: the 16-bit accumulators sum the looked-up bytes
 * of every group exactly (modulo 2^16). */
void fso_accumulate(const uint8_t* bits, uint32_t ncode, uint32_t P, const uint8_t* lut,
                    uint16_t* res) {
    const uint32_t rowb = P / 8;
    for (uint32_t v = 0; v < ncode; ++v) {
        uint32_t s = 0;
        const uint8_t* b = bits + (size_t)v * rowb;
        for (uint32_t g = 0; g < P / 4; ++g) {
            const uint32_t nib = (g & 1) ? (b[g / 2] >> 4) : (b[g / 2] & 15);
            s += lut[16 * g + nib];
        }
        res[v] = (uint16_t)s;
    }
}

/* qg/qg_scanner.hpp:110-136 (AVX-512 branch: the 16-bit sums are
 * sign-extended, doubled, minus sumq, converted) and 12-47:
 *   appro = (factor_dq * width) * r + fma(factor_vq, lower, triple_x + sqr_y)
 * which the reference's -Ofast build (its intrinsics are plain vector
 * arithmetic to the compiler) reassociates, where the scanner is inlined
 * into its caller, into
 *   ((r * factor_dq) * width) + fma(factor_vq, lower, triple_x + sqr_y),
 * as its compiled code shows. */
void fso_estimate(const uint16_t* res, uint32_t ncode, int32_t sumq, float width, float lower,
                  float sqr_y, const float* factors, float* appro) {
    const float* tx = factors;
    const float* fdq = factors + ncode;
    const float* fvq = factors + 2 * ncode;
    for (uint32_t i = 0; i < ncode; ++i) {
        const int32_t r = ((int32_t)(int16_t)res[i] << 1) - sumq;
        const float rf = (float)r;
        const float t = tx[i] + sqr_y;
        const float vq = fmaf(fvq[i], lower, t);
        appro[i] = (rf * fdq[i]) * width + vq;
    }
}

/* space/l2.hpp:16-35 (AVX-512): 16 lane accumulators of fma((a-b), (a-b))
 * in increasing d, the _mm512_reduce_add_ps tree, then the scalar tail. */
float fso_l2(const float* a, const float* b, uint32_t dim) {
    float acc[16];
    for (int l = 0; l < 16; ++l) acc[l] = 0.0f;
    const uint32_t mul = dim & ~15u;
    for (uint32_t d = 0; d < mul; ++d) {
        const float t = a[d] - b[d];
        acc[d % 16] = fmaf(t, t, acc[d % 16]);
    }
    for (int h = 8; h >= 1; h /= 2)
        for (int l = 0; l < h; ++l) acc[l] = acc[l] + acc[l + h];
    float r = acc[0];
    for (uint32_t d = mul; d < dim; ++d) {
        const float t = a[d] - b[d];
        r = fmaf(t, t, r);
    }
    return r;
}

/* ---- the search ---------------------------------------------------------- */

typedef struct {
    uint32_t id;
    float d;
} fs_cand;

/* utils/buffer.hpp:15-25: the first position whose distance is not below d. */
static size_t lower_pos(const fs_cand* a, size_t size, float d) {
    size_t lo = 0, len = size;
    while (len > 1) {
        const size_t half = len >> 1;
        len -= half;
        lo += (size_t)(a[lo + half - 1].d < d) * half;
    }
    return (lo < size && a[lo].d < d) ? lo + 1 : lo;
}

/* Exact visited set (the reference's HashBasedBooleanSet is exact). */
typedef struct {
    uint32_t* slot;
    uint32_t mask, n;
} vset;

static int vset_init(vset* s, uint32_t cap) {
    uint32_t c = 64;
    while (c < 2 * cap) c <<= 1;
    s->slot = (uint32_t*)malloc((size_t)c * 4);
    if (!s->slot) return -1;
    memset(s->slot, 0xFF, (size_t)c * 4);
    s->mask = c - 1;
    s->n = 0;
    return 0;
}

static int vset_grow(vset* s) {
    vset t;
    if (vset_init(&t, (s->mask + 1))) return -1;
    for (uint32_t i = 0; i <= s->mask; ++i)
        if (s->slot[i] != 0xFFFFFFFFu) {
            uint32_t h = (s->slot[i] * 2654435761u) & t.mask;
            while (t.slot[h] != 0xFFFFFFFFu) h = (h + 1) & t.mask;
            t.slot[h] = s->slot[i];
            t.n++;
        }
    free(s->slot);
    *s = t;
    return 0;
}

static int vset_get(const vset* s, uint32_t id) {
    uint32_t h = (id * 2654435761u) & s->mask;
    while (s->slot[h] != 0xFFFFFFFFu) {
        if (s->slot[h] == id) return 1;
        h = (h + 1) & s->mask;
    }
    return 0;
}

static int vset_set(vset* s, uint32_t id) {
    if (2 * (s->n + 1) > s->mask + 1 && vset_grow(s)) return -1;
    uint32_t h = (id * 2654435761u) & s->mask;
    while (s->slot[h] != 0xFFFFFFFFu) {
        if (s->slot[h] == id) return 0;
        h = (h + 1) & s->mask;
    }
    s->slot[h] = id;
    s->n++;
    return 0;
}

#define CHECKED 0x80000000u

static int search_one(const fso_index* ix, const float* q, uint32_t k, uint32_t ef,
                      uint32_t* out, int32_t* st) {
    const uint32_t P = ix->P, deg = ix->deg, dim = ix->dim;
    const uint32_t rowb = P / 8;
    float* rot = (float*)malloc(sizeof(float) * P);
    uint8_t* lut = (uint8_t*)malloc((size_t)P * 4);
    fs_cand* sb = (fs_cand*)malloc(sizeof(fs_cand) * (ef + 1));
    uint32_t* rid = (uint32_t*)calloc(k + 1, 4);
    float* rd = (float*)calloc(k + 1, 4);
    uint16_t* res = (uint16_t*)malloc(2 * (size_t)deg);
    float* appro = (float*)malloc(4 * (size_t)deg);
    vset vis;
    int rc = -1;
    if (!rot || !lut || !sb || !rid || !rd || !res || !appro || vset_init(&vis, 1024)) goto done;
    fso_rotate(q, dim, P, ix->diag, rot);
    float width, lower;
    int32_t sumq;
    fso_query_prepare(rot, P, lut, &width, &lower, &sumq);

    /* qg.hpp:261-263: the search buffer (capacity ef) starts with the entry
       point at FLT_MAX; the result buffer holds k */
    size_t size = 0, cur = 0, rsize = 0;
    sb[0].id = ix->entry;
    sb[0].d = FLT_MAX;
    size = 1;
    int32_t pops = 0, exact = 0, upd = 0;
    while (cur < size) {
        /* buffer.hpp:52-60: pop the first unchecked entry */
        const uint32_t u = sb[cur].id;
        sb[cur].id |= CHECKED;
        ++cur;
        while (cur < size && (sb[cur].id & CHECKED)) ++cur;
        ++pops;
        if (vset_get(&vis, u)) continue;
        if (vset_set(&vis, u)) goto done;
        /* qg.hpp:348-393: exact distance of the popped node, then the
           estimates of its neighbours and the buffer inserts in list order */
        const float sqr_y = fso_l2(q, ix->vectors + (size_t)u * dim, dim);
        ++exact;
        const uint8_t* codes = ix->codes + (size_t)u * deg * rowb;
        fso_accumulate(codes, deg, P, lut, res);
        fso_estimate(res, deg, sumq, width, lower, sqr_y, ix->factors + (size_t)u * 3 * deg, appro);
        const uint32_t* nb = ix->nbrs + (size_t)u * deg;
        for (uint32_t i = 0; i < deg; ++i) {
            const float d = appro[i];
            if (size == ef && d > sb[size - 1].d) continue; /* is_full */
            if (vset_get(&vis, nb[i])) continue;
            const size_t lo = lower_pos(sb, size, d);
            memmove(&sb[lo + 1], &sb[lo], (size - lo) * sizeof(fs_cand));
            sb[lo].id = nb[i];
            sb[lo].d = d;
            size += size < ef;
            cur = lo < cur ? lo : cur;
        }
        /* buffer.hpp:86-97: ResultBuffer::insert */
        if (!(rsize == k && sqr_y > rd[rsize - 1])) {
            size_t lo = 0, len = rsize;
            while (len > 1) {
                const size_t half = len >> 1;
                len -= half;
                lo += (size_t)(rd[lo + half - 1] < sqr_y) * half;
            }
            if (lo < rsize && rd[lo] < sqr_y) ++lo;
            memmove(&rid[lo + 1], &rid[lo], (rsize - lo) * 4);
            memmove(&rd[lo + 1], &rd[lo], (rsize - lo) * 4);
            rid[lo] = u;
            rd[lo] = sqr_y;
            rsize += rsize < k;
        }
    }
    /* qg.hpp:395-418: fewer than k results: scan the neighbours of each
       result id (a copy of all k + 1 slots, unfilled ones 0) with exact
       distances, until full */
    if (rsize < k) {
        uint32_t* ids = (uint32_t*)malloc(4 * (size_t)(k + 1));
        if (!ids) goto done;
        memcpy(ids, rid, 4 * (size_t)(k + 1));
        for (uint32_t t = 0; t <= k; ++t) {
            const uint32_t* nb = ix->nbrs + (size_t)ids[t] * deg;
            for (uint32_t i = 0; i < deg; ++i) {
                if (vset_get(&vis, nb[i])) continue;
                if (vset_set(&vis, nb[i])) {
                    free(ids);
                    goto done;
                }
                const float d = fso_l2(q, ix->vectors + (size_t)nb[i] * dim, dim);
                ++upd;
                if (rsize == k && d > rd[rsize - 1]) continue;
                size_t lo = 0, len = rsize;
                while (len > 1) {
                    const size_t half = len >> 1;
                    len -= half;
                    lo += (size_t)(rd[lo + half - 1] < d) * half;
                }
                if (lo < rsize && rd[lo] < d) ++lo;
                memmove(&rid[lo + 1], &rid[lo], (rsize - lo) * 4);
                memmove(&rd[lo + 1], &rd[lo], (rsize - lo) * 4);
                rid[lo] = nb[i];
                rd[lo] = d;
                rsize += rsize < k;
            }
            if (rsize == k) break;
        }
        free(ids);
    }
    memcpy(out, rid, 4 * (size_t)k);
    if (st) {
        st[0] = pops;
        st[1] = exact;
        st[2] = upd;
        st[3] = (int32_t)rsize;
    }
    rc = 0;
done:
    free(rot);
    free(lut);
    free(sb);
    free(rid);
    free(rd);
    free(res);
    free(appro);
    free(vis.slot);
    return rc;
}

int fso_search_batch(const fso_index* ix, const float* queries, int64_t m, const int32_t* k,
                     const int32_t* ef, uint32_t* ids, uint32_t kstride, int32_t* stats,
                     int nthreads) {
    int bad = 0;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 8) num_threads(nthreads) reduction(| : bad)
    for (int64_t i = 0; i < m; ++i) {
        const uint32_t ki = (uint32_t)k[i] < kstride ? (uint32_t)k[i] : kstride;
        const uint32_t ei = ef[i] > 0 ? (uint32_t)ef[i] : 1u;
        if (search_one(ix, queries + (size_t)i * ix->dim, ki, ei, ids + (size_t)i * kstride,
                       stats ? stats + 4 * i : NULL))
            bad = 1;
    }
    return bad ? -1 : 0;
}
