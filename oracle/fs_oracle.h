/* Test infrastructure: plain-C restatement of the upstream SymphonyQG query
 * path that LiteQG still carries but no longer calls: the FHT rotation, the
 * 6-bit query quantization and 4-bit FastScan lookup tables, the RaBitQ
 * codes, factors and distance estimate, and the sorted-buffer best-first
 * search with the exact re-rank of every popped node.
 *
 * Each function cites the reference lines it restates (paths inside the
 * LiteQG project). The restatement is pinned against the reference's own
 * functions, compiled from its sources into oracle/_ref (tests/test_fs_oracle.py).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it; the
 * product library never does. */
#ifndef LQG_FS_ORACLE_H
#define LQG_FS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A FastScan index: the search graph plus, per node, the RaBitQ codes and
 * factors of its neighbours relative to the node (the node is the centroid).
 *   codes   [n][deg][P/8]: neighbour j's sign bits, byte b holding the
 *           4-dimension groups 2b (low nibble) and 2b+1 (high nibble), the
 *           group's first dimension in the nibble's bit 3
 *   factors [n][3][deg]: triple_x, factor_dq, factor_vq of each neighbour */
typedef struct {
    const float* vectors;   /* [n][dim] raw FP32 vectors */
    const uint32_t* nbrs;   /* [n][deg] */
    const uint8_t* codes;   /* [n][deg][P/8] */
    const float* factors;   /* [n][3][deg] */
    const float* diag;      /* [P] rotation diagonal (+-1/sqrt(P)) */
    uint64_t n;
    uint32_t dim, P, deg, entry;
} fso_index;

/* P = 2^ceil(log2(dim)) (utils/tools.hpp:25-35, qg.hpp:183-188). */
uint32_t fso_padded_dim(uint32_t dim);

/* In-place unnormalised fast Hadamard transform of 2^logp floats. */
void fso_fht(float* buf, uint32_t logp);

/* FHTRotator::rotate (utils/rotator.hpp:89-114): dst[P] = H (diag * [src, 0]). */
void fso_rotate(const float* src, uint32_t dim, uint32_t P, const float* diag, float* dst);

/* QGQuery::query_prepare (qg/qg_query.hpp:30-45): the rotated query's range,
 * its 6-bit quantization (utils/scalar_quantize.hpp:12-58) and the packed
 * 4-bit lookup tables (quantization/fastscan_impl.hpp:258-270), P*4 bytes. */
void fso_query_prepare(const float* rot, uint32_t P, uint8_t* lut, float* width, float* lower,
                       int32_t* sumq);

/* rabitq_codes / rabitq_factors (quantization/rabitq.hpp:23-108) for the deg
 * rotated neighbours rot_nb[deg][P] of the rotated centroid rot_c[P]: sign
 * bits in the codes layout above and factors[3][deg]. Norms and inner
 * products are reduced in FP64. A neighbour equal to the centroid (zero
 * residual, where the reference divides 0 by 0) gets zero factors, so its
 * estimate is the centroid's exact distance. */
void fso_rabitq(const float* rot_nb, const float* rot_c, uint32_t deg, uint32_t P,
                uint8_t* bits, float* factors);

/* pack_codes (quantization/fastscan_impl.hpp:63-123): the codes of ncode
 * neighbours (ncode a multiple of 32) in the reference's FastScan block
 * layout, and back. */
void fso_pack_codes(const uint8_t* bits, uint32_t ncode, uint32_t P, uint8_t* packed);
void fso_unpack_codes(const uint8_t* packed, uint32_t ncode, uint32_t P, uint8_t* bits);

/* accumulate_impl (fastscan_impl.hpp:127-255): res[v] = sum over the P/4
 * groups of lut[group][nibble of v], mod 2^16. */
void fso_accumulate(const uint8_t* bits, uint32_t ncode, uint32_t P, const uint8_t* lut,
                    uint16_t* res);

/* QGScanner::scan_neighbors + appro_dist_impl (qg/qg_scanner.hpp:12-47,
 * 99-155), AVX-512 branch: the RaBitQ estimate of each neighbour. */
void fso_estimate(const uint16_t* res, uint32_t ncode, int32_t sumq, float width, float lower,
                  float sqr_y, const float* factors, float* appro);

/* search_qg (qg/qg.hpp:252-287) with scan_neighbors (:348-393), the sorted
 * SearchBuffer (utils/buffer.hpp:10-78), ResultBuffer (:80-119) and
 * update_results (qg.hpp:395-418), per query. ids[m][kstride]: the k ids the
 * reference copies out (slots it never fills hold 0, as its zero-initialised
 * buffer does). stats[m][4] (may be NULL): buffer pops, exact evaluations of
 * popped nodes, exact evaluations in update_results, final result count.
 * Returns 0, or -1 on allocation failure. */
int fso_search_batch(const fso_index* ix, const float* queries, int64_t m, const int32_t* k,
                     const int32_t* ef, uint32_t* ids, uint32_t kstride, int32_t* stats,
                     int nthreads);

/* The reference's 16-lane l2_sqr on raw FP32 vectors (space/l2.hpp:16-35). */
float fso_l2(const float* a, const float* b, uint32_t dim);

#ifdef __cplusplus
}
#endif
#endif
