// Work order of a batch: the queries expected to run longest first.
//
// The search kernels take queries from a device work queue, one per warp, as
// warps free up, so a batch ends when its last-started long queries end. A
// query's length is not known before it runs. Two cheap predictors: its ef (a
// search pops at least ef nodes), and its distance to the entry point (where
// every search starts; the farther, the longer the walk to its region). The
// order is by ef, then by that distance, both descending; on the bench's 1M
// batch it shortens the batch by 8 % (ordering by the true pop counts would
// give 24 %). The order changes no result: every query is searched alone.
#include <cub/device/device_radix_sort.cuh>

#include "lqg_host.h"
#include "lqg_internal.h"

namespace lqg {

// key[i] descends with (ef_i, |q_i - decoded entry|^2), so that an ascending
// sort puts the longest-expected queries first; idx[i] = i. One warp per
// query. Without per-query ef: key = ~bits(distance) (non-negative floats
// order as their bits). With it: ~(min(ef, 1023) << 22 | bits(distance) >> 10).
__global__ void entry_distance_kernel(const float* __restrict__ q, int64_t m, uint32_t dim,
                                      const uint8_t* __restrict__ ecode,
                                      const float* __restrict__ params,
                                      const uint32_t* __restrict__ efq, uint32_t* __restrict__ key,
                                      int32_t* __restrict__ idx) {
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= m) return;  // whole warps
    float s = 0.f;
    for (uint32_t d = lane; d < dim; d += 32) {
        const float dec = fmaf((float)ecode[d], params[2 * d + 1], params[2 * d]);
        const float df = q[(size_t)i * dim + d] - dec;
        s = fmaf(df, df, s);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) {
        const uint32_t db = __float_as_uint(s);
        key[i] = efq ? ~((min(efq[i], 1023u) << 22) | (db >> 10)) : ~db;
        idx[i] = (int32_t)i;
    }
}

}  // namespace lqg

namespace lqg_host {

// Sizes the work-order buffers for chunks of up to `chunk` queries.
lqg_status ensure_order(Workspace& w, int64_t chunk) {
    lqg_status s;
    if ((s = grow(w.d_okey, w.cap_okey, (size_t)chunk * 2)) != LQG_OK) return s;
    if ((s = grow(w.d_oidx, w.cap_oidx, (size_t)chunk * 2)) != LQG_OK) return s;
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const int32_t*)nullptr, (int32_t*)nullptr, (int)chunk, 0, 32);
    return grow(w.d_otemp, w.cap_otemp, tb);
}

// The work list of queries [0, m) of `queries` (per-query ef efq or NULL):
// longest expected first, sorted on the key's top 16 bits (24 with efq).
lqg_status order_queries(const lqg_index* ix, Workspace& w, const float* queries,
                         const uint32_t* efq, int64_t m, cudaStream_t st, const int32_t** list) {
    uint32_t* kin = w.d_okey;
    uint32_t* kout = w.d_okey + w.cap_okey / 2;
    int32_t* vin = w.d_oidx;
    int32_t* vout = w.d_oidx + w.cap_oidx / 2;
    const int threads = 256;
    const int64_t blocks = (m * 32 + threads - 1) / threads;
    lqg::entry_distance_kernel<<<(unsigned)blocks, threads, 0, st>>>(
        queries, m, ix->dim, ix->d_codes + (size_t)ix->entry * ix->cstride, ix->d_params, efq, kin,
        vin);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "work-order launch");
    size_t tb = w.cap_otemp;
    e = cub::DeviceRadixSort::SortPairs(w.d_otemp, tb, kin, kout, vin, vout, (int)m,
                                        efq ? 8 : 16, 32, st);
    if (e != cudaSuccess) return cuda_fail(e, "work-order sort");
    *list = vout;
    return LQG_OK;
}

}  // namespace lqg_host
