/* Test infrastructure only: a plain-C restatement of the reference's
 * quantized-graph query path (LiteQG, symqglib/qg/qg.hpp:298-344), used by
 * tests/ and bench.py's CPU baseline as the checker. The product library never
 * links or calls it.
 *
 * Index arrays (split out of the reference's file layout, qg.hpp:206-224):
 *   nbrs   [n][deg] uint32   neighbour ids of each node
 *   codes  [n][dim] uint8    SQ8 codes
 *   params [dim][2] float    (min, scale) per dimension
 */
#ifndef LQG_ORACLE_H
#define LQG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const uint32_t* nbrs;
    const uint8_t* codes;
    const float* params;
    uint64_t n;
    uint32_t dim;
    uint32_t deg;
    uint32_t entry;
    int lanes; /* 16: reference built with AVX-512; 8: AVX2 */
} lqgo_index;

/* SQ8 decode + squared L2 in the reference's summation order. */
float lqgo_sq8_l2(const float* q, const uint8_t* code, const float* params,
                  uint32_t dim, int lanes);

/* SQ8 encoder (sq8.hpp:11-26). recip bit 1: scale = (max-min) * (1/255), as
 * the reference's -Ofast build computes it (pinned against it); bit 0: the
 * per-value division by scale becomes a multiply by 1/scale (not what the
 * reference does; kept to show the difference). Use recip = 2. */
void lqgo_sq8_quantize(const float* data, uint64_t dim, uint64_t n,
                       uint8_t* codes, float* params, int recip);

/* One query. compat[k] receives exactly what the reference search() writes;
 * slots it leaves unwritten are set to 0xFFFFFFFF. pool_ids/pool_d[ef]
 * receive the final result pool in ascending order (the reverse of the
 * reference's pop order); *pool_n its size. pops/evals count heap pops and
 * neighbour distance evaluations. Returns 0, or -1 on allocation failure. */
int lqgo_search(const lqgo_index* ix, const float* q, int k, int ef,
                uint32_t* compat, uint32_t* pool_ids, float* pool_d,
                int* pool_n, int* pops, int* evals);

/* M queries with per-query k and ef (arrays, or NULL to use k0/ef0).
 * Output strides: compat kmax per query, pool efmax per query.
 * pool_ids/pool_d/pool_n/pops/evals may be NULL. nthreads <= 0: all. */
int lqgo_search_batch(const lqgo_index* ix, const float* q, int64_t m,
                      const int* k, int k0, const int* ef, int ef0, int kmax,
                      int efmax, uint32_t* compat, uint32_t* pool_ids,
                      float* pool_d, int* pool_n, int* pops, int* evals,
                      int nthreads);

#ifdef __cplusplus
}
#endif
#endif
