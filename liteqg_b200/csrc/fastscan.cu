// FastScan / RaBitQ search path: the upstream SymphonyQG query that this
// LiteQG fork still carries but no longer calls (QuantizedGraph::search_qg,
// symqglib/qg/qg.hpp:252-287, with scan_neighbors :348-393 and
// update_results :395-418), rebuilt for sm_100a, plus the encoder that writes
// the per-node RaBitQ codes and factors the fork's builder never writes
// (quantization/rabitq.hpp:23-108, around each node as the centroid).
//
// Device layout (one contiguous row per node, so a popped node costs ONE bulk
// copy: upstream's "raw vector + packed codes + factors + neighbours" row,
// qg.hpp:73-81, with the codes neighbour-major):
//   [0, 4*D4)               f32 raw vector (D4 = D rounded up to 4)
//   [off_codes, +deg*P/8)   neighbour j's sign bits, P/8 bytes; byte b holds
//                           the 4-dimension groups 2b (low nibble) and 2b+1
//                           (high nibble), the group's first dimension on bit 3
//   [off_fac, +12*deg)      f32 triple_x[deg], factor_dq[deg], factor_vq[deg]
//   [off_ids, +4*deg)       u32 neighbour ids
// The file keeps upstream's FastScan block layout for the codes
// (fastscan_impl.hpp:63-123); rows are converted on upload.
//
// Search: one warp per query, persistent over a work queue. Per query the
// warp rotates the query (FHT, the reference's butterfly order), quantizes it
// to 6 bits and builds the 4-bit lookup tables in shared memory
// (qg_query.hpp:30-45). Per pop it copies the popped node's row into shared
// memory with one cp.async.bulk (completion on an mbarrier), asks L2 for the
// row of the next unchecked node (cp.async.bulk.prefetch), computes the exact
// L2 of the popped node (the reference's 16-lane order), accumulates the
// lookup tables over every neighbour's code (lane = neighbour, 16-bit sums),
// forms the RaBitQ estimates, and inserts the unvisited neighbours into the
// sorted search buffer (utils/buffer.hpp:10-78) in list order - all of them
// at once, from counts, exactly as the sequential inserts would.
//
// Every operation on floats restates the reference's compiled -Ofast AVX-512
// code (pinned against it in tests/test_fs_oracle.py): the query range and
// its folded reciprocal, the rounding of the quantizer, the sign-extended
// 16-bit accumulators and the reassociated estimator.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/lqg.h"
#include "lqg_host.h"
#include "lqg_kernels.cuh"

namespace lqg {

namespace {

constexpr uint32_t kChecked = 0x80000000u;
constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr uint32_t kFsErrVisited = 1u;   // a visited table filled up at its largest size
constexpr uint32_t kFsErrCopy = 2u;      // a row copy did not complete in time
constexpr uint32_t kFsErrNonFinite = 4u; // an estimate or distance was not finite

struct FsSearchArgs {
    const unsigned char* rows;
    uint64_t row_bytes;
    uint32_t n, dim, P, deg, entry;
    uint32_t off_codes, off_fac, off_ids;
    const float* diag;
    const float* queries;
    int64_t m;
    const int32_t* qlist;    // work list (NULL: 0..m-1)
    const uint32_t* nlist;   // if set, the work list length is *nlist
    const uint32_t* kq;
    uint32_t k0;
    const uint32_t* efq;
    uint32_t ef0;
    uint32_t* ids;
    uint32_t kstride;
    uint32_t* stats;         // [m][4] or NULL
    uint32_t* qhead;
    uint32_t* err;           // [0] error bits, [1] first failing query
    int32_t* retry;          // queries whose visited table filled up
    uint32_t* nretry;
    uint32_t vbits;          // visited table: 2^vbits slots
    uint32_t efcap, kcap;    // buffer capacities (ef <= efcap, k <= kcap)
    uint32_t final_round;    // a full visited table fails the query instead of a retry
};

__host__ __device__ inline uint32_t al16(uint64_t x) { return (uint32_t)((x + 15) & ~15ull); }

struct FsWarpLayout {
    uint32_t row, bar, qs, lut, sb_a, sb_b, rb, rcopy, vis, total;
};

__host__ __device__ inline FsWarpLayout fs_layout(uint32_t dim, uint32_t P, uint64_t row_bytes,
                                                  uint32_t efcap, uint32_t kcap, uint32_t vbits) {
    FsWarpLayout L;
    uint32_t o = 0;
    L.row = o;
    o += al16(row_bytes);
    L.bar = o;
    o += 16;
    L.qs = o;
    o += al16(4ull * ((dim + 15) & ~15u));
    L.lut = o;
    o += al16(4ull * P);
    L.sb_a = o;
    o += al16(8ull * (efcap + 1));
    L.sb_b = o;
    o += al16(8ull * (efcap + 1));
    L.rb = o;
    o += al16(8ull * (kcap + 1));
    L.rcopy = o;
    o += al16(4ull * (kcap + 1));
    L.vis = o;
    o += al16(4ull << vbits);
    L.total = o;
    return L;
}

// ---- async copies (bulk copy engine) --------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One elected lane: expect `bytes` on the barrier and start the copy.
__device__ __forceinline__ void bulk_row_copy(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Waits for the barrier's phase `parity` to complete; gives up after a bounded
// number of tries (each try_wait suspends for a hardware-defined time).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < (1u << 22); ++i) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// The kernel-side failure path of every bounded wait in this library, made
// to run out on purpose: an mbarrier that nothing arrives on is waited for
// `tries` times; the kernel reports the timeout in *out and returns, leaving
// the context usable.
__global__ void wait_selftest_kernel(uint32_t tries, uint32_t* out) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar);
    __syncwarp();
    bool done = false;
    for (uint32_t i = 0; i < tries && !done; ++i) {
        uint32_t d;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.u32 %0, 1, 0, p;\n}"
            : "=r"(d)
            : "r"(smem_addr(&bar)), "r"(0u)
            : "memory");
        done = d != 0;
    }
    if (threadIdx.x == 0) *out = done ? 0u : 1u;
}

__device__ __forceinline__ void l2_prefetch_row(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// ---- exact visited set: open addressing in shared memory -------------------

__device__ __forceinline__ uint32_t vhash(uint32_t id, uint32_t vbits) {
    return (id * 0x9E3779B1u) >> (32u - vbits);
}

// Lane-private probe: is `id` in the set?
__device__ __forceinline__ bool vis_has(const uint32_t* vis, uint32_t vbits, uint32_t id) {
    const uint32_t mask = (1u << vbits) - 1;
    uint32_t h = vhash(id, vbits);
    for (uint32_t t = 0; t <= mask; ++t) {
        const uint32_t s = vis[h];
        if (s == id) return true;
        if (s == kEmpty) return false;
        h = (h + 1) & mask;
    }
    return false;
}

// Warp-wide test-and-insert of one id (every lane passes the same id).
// Returns true when it was already present. The caller keeps the count and
// stops at half occupancy, so an empty slot always exists.
__device__ __forceinline__ bool vis_test_insert(uint32_t* vis, uint32_t vbits, uint32_t id,
                                                int lane) {
    const uint32_t mask = (1u << vbits) - 1;
    uint32_t h0 = vhash(id, vbits);
    for (uint32_t base = 0; base <= mask; base += 32) {
        const uint32_t s = vis[(h0 + base + lane) & mask];
        const unsigned hit = __ballot_sync(kFull, s == id);
        const unsigned emp = __ballot_sync(kFull, s == kEmpty);
        if (hit && (!emp || __ffs(hit) < __ffs(emp))) return true;
        if (emp) {
            __syncwarp();
            if (lane == 0) vis[(h0 + base + __ffs(emp) - 1) & mask] = id;
            __syncwarp();
            return false;
        }
    }
    return false;
}

// ---- the exact distance ----------------------------------------------------

// space/l2.hpp:16-35: lanes 0-15 own accumulator l (dimensions l, l+16, ...,
// in increasing order), the _mm512_reduce_add_ps fold tree across them, then
// the scalar tail for dim % 16. Result in every lane.
__device__ __forceinline__ float exact_l2(const float* q, const float* v, uint32_t dim, int lane) {
    const uint32_t mul = dim & ~15u;
    float acc = 0.f;
    if (lane < 16)
        for (uint32_t d = lane; d < mul; d += 16) {
            const float t = __fsub_rn(q[d], v[d]);
            acc = __fmaf_rn(t, t, acc);
        }
    acc = __fadd_rn(acc, __shfl_down_sync(kFull, acc, 8));
    acc = __fadd_rn(acc, __shfl_down_sync(kFull, acc, 4));
    acc = __fadd_rn(acc, __shfl_down_sync(kFull, acc, 2));
    acc = __fadd_rn(acc, __shfl_down_sync(kFull, acc, 1));
    float r = __shfl_sync(kFull, acc, 0);
    for (uint32_t d = mul; d < dim; ++d) {
        const float t = __fsub_rn(q[d], v[d]);
        r = __fmaf_rn(t, t, r);
    }
    return r;
}

// Number of entries of the ascending d[0, n) strictly below y.
__device__ __forceinline__ uint32_t count_below(const float* d, uint32_t n, float y) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (d[mid] < y)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// ResultBuffer::insert (utils/buffer.hpp:86-97): capacity k; a distance above
// the last of a full buffer is dropped; otherwise it goes before the equal
// ones and the last falls off. Warp-wide.
__device__ __forceinline__ void result_insert(float* rd, uint32_t* ri, uint32_t& rsize, uint32_t k,
                                              uint32_t id, float y, int lane) {
    if (k == 0 || (rsize == k && y > rd[rsize - 1])) return;
    const uint32_t pos = count_below(rd, rsize, y);
    // shift [pos, rsize) up by one (into the k + 1 slots), from the top
    for (int base = (int)((rsize - 1) & ~31u); rsize > pos && base >= (int)(pos & ~31u); base -= 32) {
        const uint32_t x = (uint32_t)base + lane;
        float dv = 0.f;
        uint32_t iv = 0;
        const bool mv = x >= pos && x < rsize;
        if (mv) {
            dv = rd[x];
            iv = ri[x];
        }
        __syncwarp();
        if (mv) {
            rd[x + 1] = dv;
            ri[x + 1] = iv;
        }
        __syncwarp();
    }
    if (lane == 0) {
        rd[pos] = y;
        ri[pos] = id;
    }
    __syncwarp();
    rsize += rsize < k ? 1u : 0u;
}

template <int DEGW>
__global__ void __launch_bounds__(256, 4) fs_search_kernel(FsSearchArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t dim = a.dim, P = a.P, deg = a.deg;
    const FsWarpLayout L = fs_layout(dim, P, a.row_bytes, a.efcap, a.kcap, a.vbits);
    unsigned char* wb = smem + (size_t)warp * L.total;
    unsigned char* row = wb + L.row;
    uint64_t* bar = reinterpret_cast<uint64_t*>(wb + L.bar);
    float* qs = reinterpret_cast<float*>(wb + L.qs);
    uint8_t* lut = wb + L.lut;
    float* sbd[2] = {reinterpret_cast<float*>(wb + L.sb_a), reinterpret_cast<float*>(wb + L.sb_b)};
    uint32_t* sbi[2] = {reinterpret_cast<uint32_t*>(sbd[0] + (a.efcap + 1)),
                        reinterpret_cast<uint32_t*>(sbd[1] + (a.efcap + 1))};
    float* rd = reinterpret_cast<float*>(wb + L.rb);
    uint32_t* ri = reinterpret_cast<uint32_t*>(rd + (a.kcap + 1));
    uint32_t* rcopy = reinterpret_cast<uint32_t*>(wb + L.rcopy);
    uint32_t* vis = reinterpret_cast<uint32_t*>(wb + L.vis);
    const uint32_t vhalf = 1u << (a.vbits - 1);
    const uint32_t PB = P / 8;
    const int64_t mlist = a.nlist ? (int64_t)*a.nlist : a.m;
    uint32_t logp = 0;
    while ((1u << logp) < P) ++logp;

    if (lane == 0) mbar_init(bar);
    __syncwarp();
    uint32_t phase = 0;

    for (;;) {
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(a.qhead, 1u);
        slot = __shfl_sync(kFull, slot, 0);
        if ((int64_t)slot >= mlist) break;
        const int64_t qi = a.qlist ? (int64_t)a.qlist[slot] : (int64_t)slot;
        uint32_t ef = a.efq ? a.efq[qi] : a.ef0;
        ef = min(max(ef, 1u), a.efcap);
        const uint32_t k = min(min(a.kq ? a.kq[qi] : a.k0, a.kstride), a.kcap);
        const float* q = a.queries + (size_t)qi * dim;

        // ---- query preparation (qg_query.hpp:30-45) ----
        float* rot = reinterpret_cast<float*>(row);  // the row buffer is free here
        for (uint32_t i = lane; i < P; i += 32) {
            const float v = i < dim ? q[i] : 0.f;
            if (i < ((dim + 15) & ~15u)) qs[i] = v;
            rot[i] = i < dim ? __fmul_rn(v, a.diag[i]) : 0.f;
        }
        for (uint32_t i = P + lane; i < ((dim + 15) & ~15u); i += 32) qs[i] = 0.f;
        __syncwarp();
        // the FHT: butterflies on the lowest index bit first (third/ffht)
        for (uint32_t s = 0; s < logp; ++s) {
            const uint32_t h = 1u << s;
            for (uint32_t t = lane; t < P / 2; t += 32) {
                const uint32_t j = ((t >> s) << (s + 1)) | (t & (h - 1));
                const float x = rot[j], y = rot[j + h];
                rot[j] = __fadd_rn(x, y);
                rot[j + h] = __fsub_rn(x, y);
            }
            __syncwarp();
        }
        // range with the vector min/max starting from zero (scalar_quantize.hpp:12-37)
        float lo = 0.f, hi = 0.f;
        for (uint32_t i = lane; i < P; i += 32) {
            const float v = rot[i];
            lo = v < lo ? v : lo;
            hi = v > hi ? v : hi;
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(kFull, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(kFull, hi, o));
        }
        const float range = __fsub_rn(hi, lo);
        // width = range * fl(1/63); 1 / width folded into fl(1/fl(1/63)) / range
        const float width = __fmul_rn(range, __uint_as_float(0x3C820821u));
        const float inv = __fdiv_rn(__uint_as_float(0x427BFFFFu), range);
        int32_t sumq = 0;
        uint8_t* bq = reinterpret_cast<uint8_t*>(rot);  // byte i overwrites float i/4: read first
        for (uint32_t base = 0; base < P; base += 128) {
            uint32_t qv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t i = base + u * 32 + lane;
                uint32_t b = 0;
                if (i < P) {
                    const float t = __fmul_rn(__fsub_rn(rot[i], lo), inv);
                    // std::lround as compiled: trunc((t + 0.5) + 0.49999999999999994),
                    // a NaN (zero range) converts to the x86 integer indefinite
                    const double x = __dadd_rn(__dadd_rn((double)t, 0.5), 0.49999999999999994);
                    b = (t == t) ? (uint32_t)(long long)trunc(x) & 0xFFu : 0u;
                }
                qv[u] = b;
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t i = base + u * 32 + lane;
                if (i < P) {
                    bq[i] = (uint8_t)qv[u];
                    sumq += (int32_t)qv[u];
                }
            }
            __syncwarp();
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) sumq += __shfl_xor_sync(kFull, sumq, o);
        // lookup tables (fastscan_impl.hpp:258-270): group g, nibble j: the sum
        // of the group's bytes whose bit is set in j, bit 3 = the group's first
        for (uint32_t g = lane; g < P / 4; g += 32) {
            const uint32_t b0 = bq[4 * g], b1 = bq[4 * g + 1], b2 = bq[4 * g + 2], b3 = bq[4 * g + 3];
            uint32_t w[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                uint32_t word = 0;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int j = 4 * c + e;
                    const uint32_t v = ((j & 8) ? b0 : 0u) + ((j & 4) ? b1 : 0u) +
                                       ((j & 2) ? b2 : 0u) + ((j & 1) ? b3 : 0u);
                    word |= (v & 0xFFu) << (8 * e);
                }
                w[c] = word;
            }
            *reinterpret_cast<uint4*>(lut + 16 * g) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        for (uint32_t i = lane; i < (1u << a.vbits); i += 32) vis[i] = kEmpty;
        __syncwarp();

        // ---- search_qg (qg.hpp:252-287) ----
        int cb = 0;  // current sorted buffer
        float* sd = sbd[0];
        uint32_t* si = sbi[0];
        if (lane == 0) {
            sd[0] = CUDART_MAX_NORMAL_F;  // FLT_MAX
            si[0] = a.entry;
        }
        __syncwarp();
        uint32_t size = 1, cur = 0, rsize = 0, nvis = 0;
        uint32_t pops = 0, exact = 0, upd = 0;
        bool fail = false, overflow = false;

        while (cur < size && !fail) {
            // SearchBuffer::pop (buffer.hpp:52-60)
            const uint32_t u = si[cur];
            __syncwarp();
            if (lane == 0) si[cur] = u | kChecked;
            __syncwarp();
            {
                uint32_t nxt = size;
                for (uint32_t x0 = cur + 1; x0 < size; x0 += 32) {
                    const uint32_t x = x0 + lane;
                    const unsigned um = __ballot_sync(kFull, x < size && !(si[x] & kChecked));
                    if (um) {
                        nxt = x0 + __ffs(um) - 1;
                        break;
                    }
                }
                cur = nxt;
            }
            ++pops;
            if (vis_test_insert(vis, a.vbits, u, lane)) continue;
            if (++nvis >= vhalf) {
                overflow = true;
                break;
            }
            // the next unchecked node is the likely next pop: ask L2 for its row
            if (lane == 0 && cur < size)
                l2_prefetch_row(a.rows + (size_t)si[cur] * a.row_bytes, (uint32_t)a.row_bytes);
            // the popped node's row into shared memory
            __syncwarp();
            if (lane == 0)
                bulk_row_copy(row, a.rows + (size_t)u * a.row_bytes, (uint32_t)a.row_bytes, bar);
            if (!mbar_wait(bar, phase)) {
                // the copy never completed: report, wait once more, give up the warp
                if (lane == 0) {
                    atomicOr(a.err, kFsErrCopy);
                    atomicCAS(a.err + 1, kNoId, (uint32_t)qi);
                }
                mbar_wait(bar, phase);
                return;
            }
            phase ^= 1u;
            const float* vec = reinterpret_cast<const float*>(row);
            const uint8_t* codes = row + a.off_codes;
            const float* fac = reinterpret_cast<const float*>(row + a.off_fac);
            const uint32_t* nid = reinterpret_cast<const uint32_t*>(row + a.off_ids);

            // scan_neighbors (qg.hpp:348-393): exact distance of the popped node
            const float sqr_y = exact_l2(qs, vec, dim, lane);
            ++exact;
            // estimates of every neighbour (qg_scanner.hpp:99-155): lane = neighbour
            float y[DEGW];
            uint32_t id[DEGW];
            bool cand[DEGW];
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                const uint32_t j = w * 32 + lane;
                const uint8_t* c = codes + (size_t)j * PB;
                uint32_t s = 0;
                for (uint32_t c0 = 0; c0 < PB; c0 += 16) {
                    uint32_t cw[4];
                    if (PB >= 16) {
                        const uint4 v = *reinterpret_cast<const uint4*>(c + c0);
                        cw[0] = v.x;
                        cw[1] = v.y;
                        cw[2] = v.z;
                        cw[3] = v.w;
                    } else {
                        const uint2 v = *reinterpret_cast<const uint2*>(c + c0);
                        cw[0] = v.x;
                        cw[1] = v.y;
                        cw[2] = cw[3] = 0;
                    }
                    const uint8_t* lg = lut + 32 * c0;  // group 2 * c0
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        if (PB < 16 && e >= 2) break;
#pragma unroll
                        for (int bi = 0; bi < 4; ++bi) {
                            const uint32_t byte = (cw[e] >> (8 * bi)) & 0xFFu;
                            const uint8_t* gl = lg + 32 * (4 * e + bi);
                            s += gl[byte & 15u] + gl[16 + (byte >> 4)];
                        }
                    }
                }
                // 16-bit sums, sign-extended, doubled, minus sumq (qg_scanner.hpp:110-136)
                const int32_t r = ((int32_t)(int16_t)(uint16_t)(s & 0xFFFFu) << 1) - sumq;
                const float rf = __int2float_rn(r);
                const float tx = fac[j], fdq = fac[deg + j], fvq = fac[2 * deg + j];
                const float vq = __fmaf_rn(fvq, lo, __fadd_rn(tx, sqr_y));
                y[w] = __fadd_rn(__fmul_rn(__fmul_rn(rf, fdq), width), vq);
                id[w] = nid[j];
            }
            __syncwarp();  // the row buffer is read; the next copy may overwrite it
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                cand[w] = !vis_has(vis, a.vbits, id[w]);
                if (cand[w] && !(fabsf(y[w]) <= CUDART_MAX_NORMAL_F)) fail = true;
            }
            if (__any_sync(kFull, fail) || !(fabsf(sqr_y) <= CUDART_MAX_NORMAL_F)) {
                if (lane == 0) {
                    atomicOr(a.err, kFsErrNonFinite);
                    atomicCAS(a.err + 1, kNoId, (uint32_t)qi);
                }
                fail = true;
                break;
            }
            // Inserts in list order (qg.hpp:375-390): candidate j (unvisited)
            // goes in exactly when fewer than ef of everything inserted so far
            // lies strictly below it; the buffer holds the ef smallest of
            // those, so that is #{buffer < y_j} + #{earlier candidates < y_j}.
            uint32_t below[DEGW], pc[DEGW];
            bool acc[DEGW];
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                // a full buffer whose largest value lies below y_j already
                // holds ef values under it: j cannot go in, and it lies above
                // every candidate that can, so it counts for none of them
                cand[w] = cand[w] && (size < ef || y[w] <= sd[size - 1]);
                below[w] = cand[w] ? count_below(sd, size, y[w]) : 0u;
            }
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                uint32_t c = 0;
#pragma unroll
                for (int w2 = 0; w2 <= w; ++w2) {
                    unsigned bm = __ballot_sync(kFull, cand[w2]);  // warp-uniform loop
                    while (bm) {
                        const int s = __ffs(bm) - 1;
                        bm &= bm - 1;
                        const float ys = __shfl_sync(kFull, y[w2], s);
                        c += ((w2 < w || s < lane) && ys < y[w]) ? 1u : 0u;
                    }
                }
                pc[w] = c;
                acc[w] = cand[w] && below[w] + c < ef;
            }
            unsigned am[DEGW];
            uint32_t m = 0;
#pragma unroll
            for (int w = 0; w < DEGW; ++w) {
                am[w] = __ballot_sync(kFull, acc[w]);
                m += __popc(am[w]);
            }
            if (m > 0) {
                // merged order: distance ascending; an inserted value goes
                // before equal ones already there, so later candidates first
                uint32_t pos[DEGW];
#pragma unroll
                for (int w = 0; w < DEGW; ++w) {
                    uint32_t c = 0;
#pragma unroll
                    for (int w2 = 0; w2 < DEGW; ++w2) {
                        unsigned bm = am[w2];
                        while (bm) {
                            const int s = __ffs(bm) - 1;
                            bm &= bm - 1;
                            const float ys = __shfl_sync(kFull, y[w2], s);
                            const int js = w2 * 32 + s, jj = w * 32 + lane;
                            c += (ys < y[w] || (ys == y[w] && js > jj)) ? 1u : 0u;
                        }
                    }
                    pos[w] = below[w] + c;
                }
                float* nd = sbd[cb ^ 1];
                uint32_t* ni = sbi[cb ^ 1];
                const uint32_t nsize = min(size + m, ef);
                uint32_t ncur = kEmpty;
                // the old entries move up by the inserted values at or below them
                for (uint32_t x0 = 0; x0 < size; x0 += 32) {
                    const uint32_t x = x0 + lane;
                    float dx = 0.f;
                    uint32_t ix = 0, sh = 0;
                    if (x < size) {
                        dx = sd[x];
                        ix = si[x];
                    }
#pragma unroll
                    for (int w2 = 0; w2 < DEGW; ++w2) {
                        unsigned bm = am[w2];
                        while (bm) {
                            const int s = __ffs(bm) - 1;
                            bm &= bm - 1;
                            sh += __shfl_sync(kFull, y[w2], s) <= dx ? 1u : 0u;
                        }
                    }
                    const uint32_t np = x + sh;
                    if (x < size && np < nsize) {
                        nd[np] = dx;
                        ni[np] = ix;
                        if (!(ix & kChecked)) ncur = min(ncur, np);
                    }
                }
#pragma unroll
                for (int w = 0; w < DEGW; ++w)
                    if (acc[w] && pos[w] < nsize) {
                        nd[pos[w]] = y[w];
                        ni[pos[w]] = id[w];
                        ncur = min(ncur, pos[w]);
                    }
                ncur = __reduce_min_sync(kFull, ncur);
                __syncwarp();
                cb ^= 1;
                sd = nd;
                si = ni;
                size = nsize;
                cur = min(ncur, size);
            }
            // ResultBuffer::insert of the popped node (qg.hpp:285)
            result_insert(rd, ri, rsize, k, u, sqr_y, lane);
        }

        // update_results (qg.hpp:395-418): fewer than k results
        if (!fail && !overflow && rsize < k) {
            for (uint32_t t = lane; t <= k; t += 32) rcopy[t] = t < rsize ? ri[t] : 0u;
            __syncwarp();
            for (uint32_t t = 0; t <= k && rsize < k && !overflow; ++t) {
                const unsigned char* nrow = a.rows + (size_t)rcopy[t] * a.row_bytes;
                const uint32_t* nb = reinterpret_cast<const uint32_t*>(nrow + a.off_ids);
                for (uint32_t i = 0; i < deg; ++i) {
                    const uint32_t v = nb[i];
                    if (vis_test_insert(vis, a.vbits, v, lane)) continue;
                    if (++nvis >= vhalf) {
                        overflow = true;
                        break;
                    }
                    const float d = exact_l2(qs, reinterpret_cast<const float*>(
                                                     a.rows + (size_t)v * a.row_bytes),
                                             dim, lane);
                    ++upd;
                    result_insert(rd, ri, rsize, k, v, d, lane);
                }
            }
        }
        if (overflow && !a.final_round) {
            if (lane == 0) a.retry[atomicAdd(a.nretry, 1u)] = (int32_t)qi;
            continue;
        }
        if (overflow) {
            if (lane == 0) {
                atomicOr(a.err, kFsErrVisited);
                atomicCAS(a.err + 1, kNoId, (uint32_t)qi);
            }
            fail = true;
        }
        uint32_t* out = a.ids + (size_t)qi * a.kstride;
        // copy_results (buffer.hpp:108): all k slots; never-filled ones hold 0
        for (uint32_t t = lane; t < k; t += 32) out[t] = fail ? kNoId : (t < rsize ? ri[t] : 0u);
        if (a.stats && lane == 0)
            *reinterpret_cast<uint4*>(a.stats + 4 * (size_t)qi) = make_uint4(pops, exact, upd, rsize);
        __syncwarp();
    }
}

// ---- encoder: rotation, RaBitQ codes and factors ----------------------------

// rot[i][P] = H (diag * [x_i, 0]) (utils/rotator.hpp:89-114), one warp per vector.
__global__ void fs_rotate_kernel(const float* x, uint64_t n, uint32_t dim, uint32_t P,
                                 const float* diag, float* rot) {
    extern __shared__ float sbuf[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* s = sbuf + (size_t)warp * P;
    uint32_t logp = 0;
    while ((1u << logp) < P) ++logp;
    for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp; i < n;
         i += (uint64_t)gridDim.x * (blockDim.x >> 5)) {
        const float* xi = x + i * dim;
        for (uint32_t d = lane; d < P; d += 32) s[d] = d < dim ? __fmul_rn(xi[d], diag[d]) : 0.f;
        __syncwarp();
        for (uint32_t st = 0; st < logp; ++st) {
            const uint32_t h = 1u << st;
            for (uint32_t t = lane; t < P / 2; t += 32) {
                const uint32_t j = ((t >> st) << (st + 1)) | (t & (h - 1));
                const float a = s[j], b = s[j + h];
                s[j] = __fadd_rn(a, b);
                s[j + h] = __fsub_rn(a, b);
            }
            __syncwarp();
        }
        for (uint32_t d = lane; d < P; d += 32) rot[i * P + d] = s[d];
        __syncwarp();
    }
}

// quantization/rabitq.hpp:23-108 for every (node, neighbour): the residual of
// the rotated neighbour around the rotated node, its sign bits, and the three
// factors with the norm and inner products reduced in FP64. One warp per
// (node, neighbour); writes the device row's code and factor slots.
__global__ void fs_encode_kernel(const float* rot, const uint32_t* nbrs, uint64_t n, uint32_t P,
                                 uint32_t deg, unsigned char* rows, uint64_t row_bytes,
                                 uint32_t off_codes, uint32_t off_fac) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double fac_norm = 1.0 / sqrt((double)P);
    const uint64_t total = n * deg;
    for (uint64_t e = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp; e < total;
         e += (uint64_t)gridDim.x * (blockDim.x >> 5)) {
        const uint64_t node = e / deg;
        const uint32_t j = (uint32_t)(e % deg);
        const float* c = rot + node * P;
        const float* o = rot + (size_t)nbrs[e] * P;
        unsigned char* rw = rows + node * row_bytes;
        double nrm2 = 0.0, dotx = 0.0, dotc = 0.0;
        int pop = 0;
        uint8_t* bits = rw + off_codes + (size_t)j * (P / 8);
        for (uint32_t d0 = 0; d0 < P; d0 += 32) {
            const uint32_t d = d0 + lane;
            const float r = __fsub_rn(o[d], c[d]);
            const bool s = r > 0.f;
            const double sg = s ? 1.0 : -1.0;
            nrm2 += (double)r * (double)r;
            dotx += (double)r * sg;
            dotc += (double)c[d] * sg;
            const unsigned bm = __ballot_sync(kFull, s);
            pop += __popc(bm);
            // bytes d0/8 .. d0/8+3: dimension 8b + t on bit 3 - t (t < 4) or 7 - (t - 4)
            if (lane < 4) {
                const uint32_t by = (bm >> (8 * lane)) & 0xFFu;
                uint32_t v = 0;
#pragma unroll
                for (int t = 0; t < 8; ++t)
                    if (by & (1u << t)) v |= t < 4 ? (1u << (3 - t)) : (1u << (7 - (t - 4)));
                bits[d0 / 8 + lane] = (uint8_t)v;
            }
        }
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            nrm2 += __shfl_xor_sync(kFull, nrm2, off);
            dotx += __shfl_xor_sync(kFull, dotx, off);
            dotc += __shfl_xor_sync(kFull, dotc, off);
        }
        if (lane == 0) {
            float* fac = reinterpret_cast<float*>(rw + off_fac);
            const double x = sqrt(nrm2);
            if (!(x > 0.0)) {
                fac[j] = 0.f;
                fac[deg + j] = 0.f;
                fac[2 * deg + j] = 0.f;
            } else {
                const double x0 = dotx * fac_norm / x;
                const double x1 = dotc * fac_norm;
                const double xx0 = x / x0;
                fac[j] = (float)(x * x + 2.0 * xx0 * x1);
                fac[deg + j] = (float)(-2.0 * xx0 * fac_norm);
                fac[2 * deg + j] = (float)(-2.0 * xx0 * fac_norm * (double)(2 * pop - (int)P));
            }
        }
    }
}

// Copies the raw vectors and neighbour ids into the rows (one block per node).
__global__ void fs_rows_base_kernel(const float* x, const uint32_t* nbrs, uint64_t n, uint32_t dim,
                                    uint32_t deg, unsigned char* rows, uint64_t row_bytes,
                                    uint32_t off_codes, uint32_t off_ids) {
    for (uint64_t i = blockIdx.x; i < n; i += gridDim.x) {
        unsigned char* rw = rows + i * row_bytes;
        float* v = reinterpret_cast<float*>(rw);
        for (uint32_t d = threadIdx.x; d < off_codes / 4; d += blockDim.x)
            v[d] = d < dim ? x[i * dim + d] : 0.f;
        uint32_t* id = reinterpret_cast<uint32_t*>(rw + off_ids);
        for (uint32_t j = threadIdx.x; j < deg; j += blockDim.x) id[j] = nbrs[i * deg + j];
    }
}

__constant__ int kPerm0Dev[16] = {0, 8, 1, 9, 2, 10, 3, 11, 4, 12, 5, 13, 6, 14, 7, 15};

// Row codes <-> upstream's FastScan blocks (fastscan_impl.hpp:63-95), per node:
// for every 32 neighbours and pair of groups, 32 bytes.
__global__ void fs_codes_kernel(unsigned char* rows, uint64_t row_bytes, uint32_t off_codes,
                                uint64_t n, uint32_t P, uint32_t deg, uint8_t* packed,
                                int to_packed) {
    const uint32_t rowb = P / 8, ncb = P / 4;
    const uint32_t per_node = deg * rowb;
    for (uint64_t i = blockIdx.x; i < n; i += gridDim.x) {
        uint8_t* bits = rows + i * row_bytes + off_codes;
        uint8_t* pk = packed + i * per_node;
        for (uint32_t t = threadIdx.x; t < per_node; t += blockDim.x) {
            // packed byte t: block blk, group pair cp, byte jj
            const uint32_t blk = t / (ncb * 16), rem = t % (ncb * 16);
            const uint32_t cp = rem / 32, jj = rem % 32;
            const uint32_t half = jj / 16, j = jj % 16;
            const uint32_t v0 = blk * 32 + kPerm0Dev[j], v1 = v0 + 16;
            const uint32_t byte = cp;  // group pair (2cp, 2cp+1) is byte cp of a code row
            if (to_packed) {
                const uint8_t a = bits[v0 * rowb + byte], b = bits[v1 * rowb + byte];
                const uint8_t na = half ? (a >> 4) : (a & 15), nb = half ? (b >> 4) : (b & 15);
                pk[t] = (uint8_t)(na | (nb << 4));
            } else {
                const uint8_t p = pk[t];
                // each code byte gets its two nibbles from two packed bytes:
                // written once from the half == 0 byte, reading its partner
                if (half == 0) {
                    const uint8_t q = pk[t + 16];
                    bits[v0 * rowb + byte] = (uint8_t)((p & 15) | ((q & 15) << 4));
                    bits[v1 * rowb + byte] = (uint8_t)((p >> 4) | ((q >> 4) << 4));
                }
            }
        }
    }
}

}  // namespace

}  // namespace lqg

// ============================================================================
// Host side
// ============================================================================

namespace lqg_host {

namespace {

constexpr uint32_t kFsMaxK = 1024;
constexpr uint32_t kFsMaxVbits = 14;

void fs_geometry(lqg_index* ix) {
    FsSection& f = ix->fs;
    f.P = 1;
    while (f.P < ix->dim) f.P <<= 1;
    const uint32_t d4 = (ix->dim + 3u) & ~3u;
    f.off_codes = 4 * d4;
    f.off_fac = f.off_codes + ix->deg * (f.P / 8);
    f.off_ids = f.off_fac + 12 * ix->deg;
    f.row_bytes = f.off_ids + 4ull * ix->deg;
}

lqg_status fs_alloc(lqg_index* ix) {
    FsSection& f = ix->fs;
    dfree(f.d_rows);
    dfree(f.d_diag);
    if (cudaMalloc(&f.d_rows, ix->n * f.row_bytes) != cudaSuccess ||
        cudaMalloc(&f.d_diag, f.P * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        dfree(f.d_rows);
        return fail(LQG_ERR_NOMEM, "device allocation of the FastScan rows failed");
    }
    return LQG_OK;
}

// Raw vectors and neighbour ids into the rows (staged through the device).
lqg_status fs_rows_base(lqg_index* ix, float** d_x_out) {
    FsSection& f = ix->fs;
    float* d_x = nullptr;
    uint32_t* d_nb = nullptr;
    if (cudaMalloc(&d_x, ix->n * ix->dim * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_nb, ix->n * ix->deg * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        dfree(d_x);
        return fail(LQG_ERR_NOMEM, "staging allocation failed");
    }
    cudaError_t e = cudaMemcpy(d_x, ix->vectors.data(), ix->n * ix->dim * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d_nb, ix->nbrs.data(), ix->n * ix->deg * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        lqg::fs_rows_base_kernel<<<4 * ix->num_sms, 128>>>(d_x, d_nb, ix->n, ix->dim, ix->deg,
                                                            f.d_rows, f.row_bytes, f.off_codes,
                                                            f.off_ids);
        e = cudaGetLastError();
    }
    cudaFree(d_nb);
    if (e != cudaSuccess) {
        cudaFree(d_x);
        return cuda_fail(e, "FastScan rows");
    }
    if (d_x_out)
        *d_x_out = d_x;
    else
        cudaFree(d_x);
    return LQG_OK;
}

// Device rows -> host copy of the codes in upstream's block layout.
lqg_status fs_download_packed(lqg_index* ix) {
    FsSection& f = ix->fs;
    const size_t per = (size_t)ix->deg * (f.P / 8);
    uint8_t* d_pk = nullptr;
    if (cudaMalloc(&d_pk, ix->n * per) != cudaSuccess) {
        cudaGetLastError();
        return fail(LQG_ERR_NOMEM, "staging allocation failed");
    }
    lqg::fs_codes_kernel<<<4 * ix->num_sms, 256>>>(f.d_rows, f.row_bytes, f.off_codes, ix->n, f.P,
                                                   ix->deg, d_pk, 1);
    cudaError_t e = cudaGetLastError();
    try {
        f.packed.resize(ix->n * per);
        f.factors.resize(ix->n * 3 * (size_t)ix->deg);
    } catch (...) {
        cudaFree(d_pk);
        return fail(LQG_ERR_NOMEM, "host allocation failed");
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(f.packed.data(), d_pk, ix->n * per, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy2D(f.factors.data(), 12 * (size_t)ix->deg, f.d_rows + f.off_fac, f.row_bytes,
                         12 * (size_t)ix->deg, ix->n, cudaMemcpyDeviceToHost);
    cudaFree(d_pk);
    return e == cudaSuccess ? LQG_OK : cuda_fail(e, "FastScan download");
}

// Host codes (upstream layout) and factors -> device rows.
lqg_status fs_upload(lqg_index* ix) {
    FsSection& f = ix->fs;
    lqg_status s;
    if ((s = fs_alloc(ix)) != LQG_OK) return s;
    if ((s = fs_rows_base(ix, nullptr)) != LQG_OK) return s;
    const size_t per = (size_t)ix->deg * (f.P / 8);
    uint8_t* d_pk = nullptr;
    if (cudaMalloc(&d_pk, ix->n * per) != cudaSuccess) {
        cudaGetLastError();
        return fail(LQG_ERR_NOMEM, "staging allocation failed");
    }
    cudaError_t e = cudaMemcpy(d_pk, f.packed.data(), ix->n * per, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        lqg::fs_codes_kernel<<<4 * ix->num_sms, 256>>>(f.d_rows, f.row_bytes, f.off_codes, ix->n,
                                                       f.P, ix->deg, d_pk, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy2D(f.d_rows + f.off_fac, f.row_bytes, f.factors.data(), 12 * (size_t)ix->deg,
                         12 * (size_t)ix->deg, ix->n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(f.d_diag, f.diag.data(), f.P * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(d_pk);
    if (e != cudaSuccess) return cuda_fail(e, "FastScan upload");
    f.ready = true;
    return LQG_OK;
}

lqg_status fs_check_batch(lqg_index* ix, const float* q, int64_t m, const uint32_t* k,
                          uint32_t k0, const uint32_t* ef, uint32_t& ef0, uint32_t* ids,
                          uint32_t kstride) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (!ix->has_data) return fail(LQG_ERR_STATE, "index has no data: load or build it first");
    if (!ix->fs.ready)
        return fail(LQG_ERR_STATE, "index has no FastScan section: call lqg_fs_build or load one");
    if (m < 0 || m > (int64_t)INT32_MAX) return fail(LQG_ERR_ARG, "bad query count");
    if (m > 0 && (!q || !ids)) return fail(LQG_ERR_ARG, "null queries or ids");
    if (kstride == 0 || kstride > kFsMaxK) return fail(LQG_ERR_ARG, "kstride must be in [1, 1024]");
    if (!k && k0 > kstride) return fail(LQG_ERR_ARG, "k exceeds kstride");
    if (!ef && ef0 == 0) {
        if (ix->ef == 0) return fail(LQG_ERR_STATE, "ef not set: call set_ef first");
        ef0 = ix->ef;
    }
    if (ef0 == 0 || ef0 > kMaxEf)
        return fail(LQG_ERR_ARG, "ef (or the per-query ef bound) must be in [1, 512]");
    return LQG_OK;
}

lqg_status fs_run(lqg_index* ix, Workspace& w, const float* q, int64_t m, const uint32_t* kq,
                  uint32_t k0, const uint32_t* efq, uint32_t ef0, uint32_t* ids, uint32_t kstride,
                  uint32_t* stats, cudaStream_t st, bool plain) {
    lqg_status s;
    if ((s = ensure_ctl(w, m)) != LQG_OK) return s;
    if ((s = reset_ctl(w, st)) != LQG_OK) return s;
    if (m == 0) return LQG_OK;
    FsSection& f = ix->fs;
    lqg::FsSearchArgs a{};
    a.rows = f.d_rows;
    a.row_bytes = f.row_bytes;
    a.n = (uint32_t)ix->n;
    a.dim = ix->dim;
    a.P = f.P;
    a.deg = ix->deg;
    a.entry = ix->entry;
    a.off_codes = f.off_codes;
    a.off_fac = f.off_fac;
    a.off_ids = f.off_ids;
    a.diag = f.d_diag;
    a.queries = q;
    a.m = m;
    a.kq = kq;
    a.k0 = k0;
    a.efq = efq;
    a.ef0 = ef0;
    a.ids = ids;
    a.kstride = kstride;
    a.stats = stats;
    a.err = w.d_ctl + kCtlErr;
    a.efcap = ef0;
    a.kcap = kstride;
    // visited table: popped nodes and, when ef < k, the neighbours
    // update_results scans; at most half full. Pops run past ef (about 1.4 ef
    // on average at ef 64, more in the tail), and a query that fills the
    // table is searched again in round 1 with one warp per block, which costs
    // the batch a whole query's latency: room for 2 ef + 64 pops
    uint32_t need = 2 * (2 * ef0 + 64);
    if (kstride > ef0) need = std::max<uint32_t>(need, 2 * (ef0 + 8 + ix->deg * (kstride + 1)));
    uint32_t vb = 8;
    while ((1u << vb) < need && vb < 12) ++vb;
    const int degw = (int)(ix->deg / 32);
    // round 0: every query with a table sized for its ef and k; round 1: the
    // queries whose table filled up, with the largest table
    const int32_t* list = nullptr;
    const uint32_t* nlist = nullptr;
    for (int round = 0; round < 2; ++round) {
        a.vbits = round == 0 ? vb : kFsMaxVbits;
        a.final_round = round == 1 || vb >= kFsMaxVbits;
        const lqg::FsWarpLayout L =
            lqg::fs_layout(a.dim, a.P, a.row_bytes, a.efcap, a.kcap, a.vbits);
        int warps = plain ? 1 : 8;
        while (warps > 1 && (size_t)warps * L.total > 100 * 1024) --warps;
        const size_t smem = (size_t)warps * L.total;
        if (smem > 227 * 1024)
            return fail(LQG_ERR_CAPACITY,
                        "FastScan work area exceeds shared memory (ef, k or D too large)");
        auto kern = degw == 1   ? lqg::fs_search_kernel<1>
                    : degw == 2 ? lqg::fs_search_kernel<2>
                    : degw == 3 ? lqg::fs_search_kernel<3>
                                : lqg::fs_search_kernel<4>;
        cudaError_t e =
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "FastScan kernel attribute");
        int occ = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, warps * 32, smem);
        if (e != cudaSuccess || occ <= 0)
            return fail(LQG_ERR_CAPACITY, "FastScan kernel cannot launch");
        int64_t blocks = plain ? 1 : (int64_t)occ * ix->num_sms;
        const int64_t need_b = (m + warps - 1) / warps;
        if (need_b < blocks) blocks = need_b;
        a.qlist = list;
        a.nlist = nlist;
        a.qhead = w.d_ctl + (round ? kCtlHeapHead : kCtlFastHead);
        a.retry = w.d_flagged;
        a.nretry = w.d_ctl + kCtlFlagged;
        if (round == 0) {
            LQG_CUDA(cudaMemsetAsync(w.d_ctl + kCtlFastHead, 0, 4, st));
            LQG_CUDA(cudaMemsetAsync(w.d_ctl + kCtlHeapHead, 0, 4, st));
            LQG_CUDA(cudaMemsetAsync(w.d_ctl + kCtlFlagged, 0, 4, st));
        }
        kern<<<(unsigned)blocks, warps * 32, smem, st>>>(a);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "FastScan search launch");
        if (a.final_round) break;
        list = w.d_flagged;  // round 1 reads the list round 0 wrote; it adds none
        nlist = w.d_ctl + kCtlFlagged;
    }
    return LQG_OK;
}

lqg_status fs_status(Workspace& w, cudaStream_t st) {
    uint32_t ctl[kCtlWords];
    LQG_CUDA(cudaMemcpyAsync(ctl, w.d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st));
    LQG_CUDA(cudaStreamSynchronize(st));
    const uint32_t e = ctl[kCtlErr];
    if (e & lqg::kFsErrCopy)
        return fail(LQG_ERR_CUDA, "a FastScan row copy did not complete (query " +
                                      std::to_string(ctl[kCtlErrQuery]) + ")");
    if (e & lqg::kFsErrNonFinite)
        return fail(LQG_ERR_ARG, "a FastScan distance was not finite (query " +
                                     std::to_string(ctl[kCtlErrQuery]) + "; its ids are LQG_NO_ID)");
    if (e & lqg::kFsErrVisited)
        return fail(LQG_ERR_CAPACITY, "a FastScan query visited more than 8192 nodes (query " +
                                          std::to_string(ctl[kCtlErrQuery]) +
                                          "; its ids are LQG_NO_ID)");
    return LQG_OK;
}

}  // namespace

// File section: "LQGFS1" magic (8 bytes), u32 P, u32 degree_bound, u32
// dimension, u32 0, f32 diag[P], then per node its neighbours' codes in
// upstream's FastScan block layout (deg * P / 8 bytes) followed by its
// factors (triple_x[deg], factor_dq[deg], factor_vq[deg]) - upstream's row
// content without the vector and ids, which the reference's part of the file
// already holds.
static const char kFsMagic[8] = {'L', 'Q', 'G', 'F', 'S', '1', 0, 0};

uint64_t fs_file_bytes(const lqg_index* ix) {
    uint32_t P = 1;
    while (P < ix->dim) P <<= 1;
    return 24 + 4ull * P + ix->n * ((uint64_t)ix->deg * (P / 8) + 12ull * ix->deg);
}

lqg_status fs_read(lqg_index* ix, FILE* f) {
    char magic[8];
    uint32_t hdr[4];
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kFsMagic, 8) != 0)
        return fail(LQG_ERR_IO, "trailing bytes are not a FastScan section");
    if (std::fread(hdr, 4, 4, f) != 4) return fail(LQG_ERR_IO, "short FastScan section header");
    fs_geometry(ix);
    FsSection& fs = ix->fs;
    if (hdr[0] != fs.P || hdr[1] != ix->deg || hdr[2] != ix->dim)
        return fail(LQG_ERR_IO, "FastScan section does not match the index's dimension/degree");
    const size_t per = (size_t)ix->deg * (fs.P / 8);
    try {
        fs.diag.resize(fs.P);
        fs.packed.resize(ix->n * per);
        fs.factors.resize(ix->n * 3 * (size_t)ix->deg);
    } catch (...) {
        return fail(LQG_ERR_NOMEM, "host allocation failed");
    }
    bool ok = std::fread(fs.diag.data(), 4, fs.P, f) == fs.P;
    for (uint64_t i = 0; ok && i < ix->n; ++i) {
        ok = std::fread(&fs.packed[i * per], 1, per, f) == per &&
             std::fread(&fs.factors[i * 3 * ix->deg], 4, 3 * ix->deg, f) == 3 * ix->deg;
    }
    if (!ok) return fail(LQG_ERR_IO, "short read of the FastScan section");
    return fs_upload(ix);
}

lqg_status fs_write(const lqg_index* ix, FILE* f) {
    const FsSection& fs = ix->fs;
    const uint32_t hdr[4] = {fs.P, ix->deg, ix->dim, 0};
    bool ok = std::fwrite(kFsMagic, 1, 8, f) == 8 && std::fwrite(hdr, 4, 4, f) == 4 &&
              std::fwrite(fs.diag.data(), 4, fs.P, f) == fs.P;
    const size_t per = (size_t)ix->deg * (fs.P / 8);
    for (uint64_t i = 0; ok && i < ix->n; ++i)
        ok = std::fwrite(&fs.packed[i * per], 1, per, f) == per &&
             std::fwrite(&fs.factors[i * 3 * ix->deg], 4, 3 * ix->deg, f) == 3 * ix->deg;
    return ok ? LQG_OK : fail(LQG_ERR_IO, "write of the FastScan section failed");
}

}  // namespace lqg_host

using namespace lqg_host;

extern "C" {

LQG_API lqg_status lqg_fs_build(lqg_index* ix, uint64_t seed) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (!ix->has_data) return fail(LQG_ERR_STATE, "index has no data: load or build it first");
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    fs_geometry(ix);
    FsSection& f = ix->fs;
    f.ready = false;
    // the rotation's diagonal: seeded +-1/sqrt(P) (utils/rotator.hpp:31-47
    // seeds from std::random_device and does not save it; here it is stored)
    f.diag.resize(f.P);
    std::mt19937_64 gen(seed);
    const float sc = 1.0f / std::sqrt((float)f.P);
    for (uint32_t i = 0; i < f.P; ++i) f.diag[i] = (gen() & 1) ? sc : -sc;
    lqg_status s;
    if ((s = fs_alloc(ix)) != LQG_OK) return s;
    float* d_x = nullptr;
    if ((s = fs_rows_base(ix, &d_x)) != LQG_OK) return s;
    float* d_rot = nullptr;
    uint32_t* d_nb = nullptr;
    cudaError_t e = cudaMemcpy(f.d_diag, f.diag.data(), f.P * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && (cudaMalloc(&d_rot, ix->n * f.P * sizeof(float)) != cudaSuccess ||
                             cudaMalloc(&d_nb, ix->n * ix->deg * sizeof(uint32_t)) != cudaSuccess)) {
        cudaGetLastError();
        cudaFree(d_x);
        dfree(d_rot);
        return fail(LQG_ERR_NOMEM, "FastScan encoder allocation failed");
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(d_nb, ix->nbrs.data(), ix->n * ix->deg * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int wpb = 4;
        lqg::fs_rotate_kernel<<<8 * ix->num_sms, 32 * wpb, wpb * f.P * sizeof(float)>>>(
            d_x, ix->n, ix->dim, f.P, f.d_diag, d_rot);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        lqg::fs_encode_kernel<<<16 * ix->num_sms, 256>>>(d_rot, d_nb, ix->n, f.P, ix->deg, f.d_rows,
                                                         f.row_bytes, f.off_codes, f.off_fac);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(d_x);
    cudaFree(d_rot);
    cudaFree(d_nb);
    if (e != cudaSuccess) return cuda_fail(e, "FastScan encoder");
    if ((s = fs_download_packed(ix)) != LQG_OK) return s;
    f.ready = true;
    return LQG_OK;
}

LQG_API lqg_status lqg_fs_set_arrays(lqg_index* ix, const float* diag, const uint8_t* packed,
                                     const float* factors) {
    if (!ix || !diag || !packed || !factors) return fail(LQG_ERR_ARG, "null argument");
    if (!ix->has_data) return fail(LQG_ERR_STATE, "index has no data: load or build it first");
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    fs_geometry(ix);
    FsSection& f = ix->fs;
    f.ready = false;
    const size_t per = (size_t)ix->deg * (f.P / 8);
    try {
        f.diag.assign(diag, diag + f.P);
        f.packed.assign(packed, packed + ix->n * per);
        f.factors.assign(factors, factors + ix->n * 3 * (size_t)ix->deg);
    } catch (...) {
        return fail(LQG_ERR_NOMEM, "host allocation failed");
    }
    return fs_upload(ix);
}

LQG_API lqg_status lqg_fs_get_arrays(const lqg_index* ix, uint32_t* padded_dim, float* diag,
                                     uint8_t* packed, float* factors) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (!ix->fs.ready) return fail(LQG_ERR_STATE, "index has no FastScan section");
    const FsSection& f = ix->fs;
    if (padded_dim) *padded_dim = f.P;
    if (diag) std::memcpy(diag, f.diag.data(), f.P * 4);
    if (packed) std::memcpy(packed, f.packed.data(), f.packed.size());
    if (factors) std::memcpy(factors, f.factors.data(), f.factors.size() * 4);
    return LQG_OK;
}

LQG_API lqg_status lqg_fs_search_batch_device(lqg_index* ix, const float* queries, int64_t m,
                                              const uint32_t* k, uint32_t k0, const uint32_t* ef,
                                              uint32_t ef0, uint32_t* ids, uint32_t kstride,
                                              uint32_t* stats, void* stream) {
    lqg_status s = fs_check_batch(ix, queries, m, k, k0, ef, ef0, ids, kstride);
    if (s != LQG_OK) return s;
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    return fs_run(ix, ix->ws, queries, m, k, k0, ef, ef0, ids, kstride, stats,
                  (cudaStream_t)stream, false);
}

LQG_API lqg_status lqg_fs_stream_status(lqg_index* ix, void* stream) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    if (!ix->ws.d_ctl) return LQG_OK;
    return fs_status(ix->ws, (cudaStream_t)stream);
}

LQG_API lqg_status lqg_fs_search_batch(lqg_index* ix, const float* queries, int64_t m,
                                       const uint32_t* k, uint32_t k0, const uint32_t* ef,
                                       uint32_t ef0, uint32_t* ids, uint32_t kstride,
                                       uint32_t* stats, void* stream) {
    uint32_t efb = ef0;
    if (ef) {
        efb = 0;
        for (int64_t i = 0; i < m; ++i) efb = std::max(efb, ef[i]);
    }
    lqg_status s = fs_check_batch(ix, queries, m, k, k0, ef, efb, ids, kstride);
    if (s != LQG_OK) return s;
    if (m == 0) return LQG_OK;
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    Workspace& w = ix->ws;
    cudaStream_t st = (cudaStream_t)stream;
    if (!st) {
        if (!ix->own_stream)
            LQG_CUDA(cudaStreamCreateWithFlags(&ix->own_stream, cudaStreamNonBlocking));
        st = ix->own_stream;
    }
    if ((s = grow(w.d_q, w.cap_q, (size_t)m * ix->dim)) != LQG_OK) return s;
    if ((s = grow(w.d_ids, w.cap_ids, (size_t)m * kstride)) != LQG_OK) return s;
    if (k && (s = grow(w.d_kq, w.cap_kq, (size_t)m)) != LQG_OK) return s;
    if (ef && (s = grow(w.d_efq, w.cap_efq, (size_t)m)) != LQG_OK) return s;
    if (stats && (s = grow(w.d_stats, w.cap_stats, (size_t)m * 4)) != LQG_OK) return s;
    LQG_CUDA(cudaMemcpyAsync(w.d_q, queries, (size_t)m * ix->dim * 4, cudaMemcpyHostToDevice, st));
    if (k) LQG_CUDA(cudaMemcpyAsync(w.d_kq, k, m * 4, cudaMemcpyHostToDevice, st));
    if (ef) LQG_CUDA(cudaMemcpyAsync(w.d_efq, ef, m * 4, cudaMemcpyHostToDevice, st));
    s = fs_run(ix, w, w.d_q, m, k ? w.d_kq : nullptr, k0, ef ? w.d_efq : nullptr, efb, w.d_ids,
               kstride, stats ? w.d_stats : nullptr, st, m == 1);
    if (s != LQG_OK) return s;
    LQG_CUDA(cudaMemcpyAsync(ids, w.d_ids, (size_t)m * kstride * 4, cudaMemcpyDeviceToHost, st));
    if (stats)
        LQG_CUDA(cudaMemcpyAsync(stats, w.d_stats, (size_t)m * 16, cudaMemcpyDeviceToHost, st));
    return fs_status(w, st);
}

LQG_API lqg_status lqg_selftest_bounded_wait(int device, uint32_t tries, uint32_t* timed_out) {
    if (!timed_out || tries == 0 || tries > (1u << 20)) return fail(LQG_ERR_ARG, "tries must be in [1, 2^20]");
    DeviceScope ds(device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    uint32_t* d = nullptr;
    LQG_CUDA(cudaMalloc(&d, sizeof(uint32_t)));
    lqg::wait_selftest_kernel<<<1, 32>>>(tries, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(timed_out, d, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? LQG_OK : cuda_fail(e, "bounded-wait self-test");
}

LQG_API lqg_status lqg_fs_search(lqg_index* ix, const float* query, uint32_t k, uint32_t* results) {
    if (!ix || !query || !results) return fail(LQG_ERR_ARG, "null argument");
    if (k == 0) return LQG_OK;
    return lqg_fs_search_batch(ix, query, 1, nullptr, k, nullptr, 0, results, k, nullptr, nullptr);
}

}  // extern "C"
