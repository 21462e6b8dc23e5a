/* Test infrastructure only (see lqg_oracle.h): the CPU oracle for the
 * quantized-graph query path. Each function cites the reference code it
 * restates (paths relative to the LiteQG project root). Compiled without
 * fast-math and without FP contraction, so every fused multiply-add below is
 * an explicit fmaf(), matching what the reference's -Ofast build emits. */
#include "lqg_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

/* ---- distance ---------------------------------------------------------- */

/* symqglib/quantization/sq8.hpp:28-32: dec[d] = min[d] + q[d]*scale[d]; the
 * reference's -Ofast build contracts this into one fused multiply-add.
 * symqglib/space/l2.hpp:16-35: 16 (AVX-512) or 8 (AVX2) lane accumulators,
 * acc[d % L] = fma(x-y, x-y, acc[d % L]) in increasing d, then the reduction
 * tree of _mm512_reduce_add_ps / reduce_add_m256 (fold the upper half onto
 * the lower half until one lane is left), then a scalar tail for dim % L. */
float lqgo_sq8_l2(const float* q, const uint8_t* code, const float* params,
                  uint32_t dim, int lanes) {
    float acc[16];
    int L = lanes == 8 ? 8 : 16;
    for (int l = 0; l < L; ++l) acc[l] = 0.0f;
    uint32_t mul = dim - (dim % (uint32_t)L);
    for (uint32_t d = 0; d < mul; ++d) {
        float dec = fmaf((float)code[d], params[2 * d + 1], params[2 * d]);
        float t = q[d] - dec;
        acc[d % (uint32_t)L] = fmaf(t, t, acc[d % (uint32_t)L]);
    }
    for (int h = L / 2; h >= 1; h /= 2)
        for (int l = 0; l < h; ++l) acc[l] = acc[l] + acc[l + h];
    float r = acc[0];
    for (uint32_t d = mul; d < dim; ++d) {
        float dec = fmaf((float)code[d], params[2 * d + 1], params[2 * d]);
        float t = q[d] - dec;
        r = fmaf(t, t, r);
    }
    return r;
}

/* symqglib/quantization/sq8.hpp:11-26. The reference's -Ofast build turns
 * the division by the constant 255 into a multiplication by its rounded
 * reciprocal (recip bit 1 selects that); the per-value division by the
 * scale stays a true division unless recip bit 0 is set. */
void lqgo_sq8_quantize(const float* data, uint64_t dim, uint64_t n,
                       uint8_t* codes, float* params, int recip) {
    for (uint64_t d = 0; d < dim; ++d) {
        float mn = data[d], mx = data[d];
        /* std::min(min, val) / std::max(max, val) (sq8.hpp:13-17) as the
         * reference's -Ofast build compiles them: minss/maxss with the new
         * value second, which returns it unless the running value is strictly
         * smaller (larger). Among equal values (-0.0 and 0.0) the LAST row's
         * is kept, and that decides the file's bytes for a zero minimum. */
        for (uint64_t i = 1; i < n; ++i) {
            float v = data[i * dim + d];
            mn = mn < v ? mn : v;
            mx = mx > v ? mx : v;
        }
        float scale = (recip & 2) ? (mx - mn) * (1.0f / 255.0f) : (mx - mn) / 255.0f;
        float inv = 1.0f / scale;
        params[2 * d] = mn;
        params[2 * d + 1] = scale;
        for (uint64_t i = 0; i < n; ++i) {
            float v = data[i * dim + d] - mn;
            float x = (recip & 1) ? v * inv : v / scale;
            codes[i * dim + d] = (uint8_t)roundf(x);
        }
    }
}

/* ---- std::priority_queue restatement ----------------------------------- */
/* The reference keeps both pools in std::priority_queue<Candidate<float>>
 * ordered by CandidateComparator (lhs.distance < rhs.distance,
 * symqglib/qg/qg.hpp:289-296). Under equal distances the pop order depends on
 * the binary-heap layout, so the oracle restates the GCC libstdc++ heap
 * algorithms it compiles to (bits/stl_heap.h, GCC 13.3): push = append +
 * sift-up with comp(parent, value); pop = move the last element into a hole
 * that first descends to a leaf along the larger child (right child unless
 * comp(right, left)), then sift-up from there. */
typedef struct {
    uint32_t id;
    float d;
} cand_t;

typedef struct {
    cand_t* a;
    size_t n, cap;
} heap_t;

static int heap_reserve(heap_t* h, size_t need) {
    if (need <= h->cap) return 0;
    size_t c = h->cap ? h->cap * 2 : 256;
    while (c < need) c *= 2;
    cand_t* p = (cand_t*)realloc(h->a, c * sizeof(cand_t));
    if (!p) return -1;
    h->a = p;
    h->cap = c;
    return 0;
}

static inline int comp(cand_t x, cand_t y) { return x.d < y.d; }

static void sift_up(cand_t* a, size_t hole, size_t top, cand_t v) {
    size_t parent = (hole - 1) / 2;
    while (hole > top && comp(a[parent], v)) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}

static int heap_push(heap_t* h, uint32_t id, float d) {
    if (heap_reserve(h, h->n + 1)) return -1;
    cand_t v = {id, d};
    h->a[h->n] = v;
    sift_up(h->a, h->n, 0, v);
    h->n++;
    return 0;
}

static void heap_pop(heap_t* h) {
    size_t size = h->n;
    if (size > 1) {
        cand_t* a = h->a;
        size_t len = size - 1; /* heap range after moving the top out */
        cand_t v = a[len];
        a[len] = a[0];
        size_t hole = 0, second = 0;
        while (second < (len - 1) / 2) {
            second = 2 * (second + 1);
            if (comp(a[second], a[second - 1])) second--;
            a[hole] = a[second];
            hole = second;
        }
        if ((len & 1) == 0 && second == (len - 2) / 2) {
            second = 2 * (second + 1);
            a[hole] = a[second - 1];
            hole = second - 1;
        }
        sift_up(a, hole, 0, v);
    }
    h->n = size - 1;
}

/* ---- search ------------------------------------------------------------ */

typedef struct {
    uint32_t* stamp; /* exact visited set: stamp[id] == cur */
    uint32_t cur;
    uint64_t n;
    heap_t sp, rp;
} scratch_t;

static int scratch_init(scratch_t* s, uint64_t n) {
    memset(s, 0, sizeof(*s));
    s->stamp = (uint32_t*)calloc(n ? n : 1, sizeof(uint32_t));
    s->n = n;
    return s->stamp ? 0 : -1;
}

static void scratch_free(scratch_t* s) {
    free(s->stamp);
    free(s->sp.a);
    free(s->rp.a);
}

/* QuantizedGraph::search_qg_with_heap, symqglib/qg/qg.hpp:298-344. */
static int search_one(const lqgo_index* ix, scratch_t* s, const float* q, int k,
                      int ef, uint32_t* compat, uint32_t* pool_ids,
                      float* pool_d, int* pool_n, int* pops, int* evals) {
    if (++s->cur == 0) { /* stamp wrap: clear once every 2^32 queries */
        memset(s->stamp, 0, s->n * sizeof(uint32_t));
        s->cur = 1;
    }
    const uint32_t cur = s->cur;
    heap_t* sp = &s->sp;
    heap_t* rp = &s->rp;
    sp->n = 0;
    rp->n = 0;
    int npop = 0, neval = 0;
    const uint32_t dim = ix->dim, deg = ix->deg;
    const size_t cap = (size_t)(ef > 0 ? ef : 0);

    uint32_t node = ix->entry; /* qg.hpp:305-311 */
    float y = lqgo_sq8_l2(q, ix->codes + (size_t)node * dim, ix->params, dim,
                          ix->lanes);
    float lower = y;
    if (heap_push(sp, node, -y) || heap_push(rp, node, y)) return -1;
    s->stamp[node] = cur;

    while (sp->n) { /* qg.hpp:313-338 */
        cand_t top = sp->a[0];
        node = top.id;
        if (-top.d > lower) break;
        heap_pop(sp);
        ++npop;
        const uint32_t* nb = ix->nbrs + (size_t)node * deg;
        for (uint32_t i = 0; i < deg; ++i) {
            uint32_t v = nb[i];
            if (s->stamp[v] == cur) continue;
            s->stamp[v] = cur;
            y = lqgo_sq8_l2(q, ix->codes + (size_t)v * dim, ix->params, dim,
                            ix->lanes);
            ++neval;
            if (rp->n < cap || lower > y) {
                if (heap_push(sp, v, -y) || heap_push(rp, v, y)) return -1;
                if (rp->n > cap) heap_pop(rp);
                lower = rp->a[0].d;
            }
        }
    }

    /* qg.hpp:340-343: results[k-1..] = successive rp tops (the worst first) */
    int pn = (int)rp->n;
    for (int i = 0; i < k; ++i) compat[i] = 0xFFFFFFFFu;
    for (int j = 0; rp->n; ++j) {
        cand_t t = rp->a[0];
        if (j < k) compat[k - 1 - j] = t.id;
        if (pool_ids) pool_ids[pn - 1 - j] = t.id;
        if (pool_d) pool_d[pn - 1 - j] = t.d;
        heap_pop(rp);
    }
    if (pool_n) *pool_n = pn;
    if (pops) *pops = npop;
    if (evals) *evals = neval;
    return 0;
}

int lqgo_search(const lqgo_index* ix, const float* q, int k, int ef,
                uint32_t* compat, uint32_t* pool_ids, float* pool_d,
                int* pool_n, int* pops, int* evals) {
    scratch_t s;
    if (scratch_init(&s, ix->n)) return -1;
    int r = search_one(ix, &s, q, k, ef, compat, pool_ids, pool_d, pool_n, pops,
                       evals);
    scratch_free(&s);
    return r;
}

int lqgo_search_batch(const lqgo_index* ix, const float* q, int64_t m,
                      const int* k, int k0, const int* ef, int ef0, int kmax,
                      int efmax, uint32_t* compat, uint32_t* pool_ids,
                      float* pool_d, int* pool_n, int* pops, int* evals,
                      int nthreads) {
    int err = 0;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : omp_get_max_threads()) reduction(| : err)
    {
        scratch_t s;
        int ok = scratch_init(&s, ix->n) == 0;
        if (!ok) err = 1;
#pragma omp for schedule(dynamic, 8)
        for (int64_t i = 0; i < m; ++i) {
            if (!ok) continue;
            int ki = k ? k[i] : k0;
            int ei = ef ? ef[i] : ef0;
            int r = search_one(
                ix, &s, q + (size_t)i * ix->dim, ki, ei,
                compat + (size_t)i * kmax,
                pool_ids ? pool_ids + (size_t)i * efmax : NULL,
                pool_d ? pool_d + (size_t)i * efmax : NULL,
                pool_n ? pool_n + i : NULL, pops ? pops + i : NULL,
                evals ? evals + i : NULL);
            if (r) err = 1;
        }
        scratch_free(&s);
    }
    return err ? -1 : 0;
}
