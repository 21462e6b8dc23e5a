// Host-side internals shared by the C-ABI implementation (lqg_api.cu) and the
// serving loop (lqg_server.cu): the index object, per-batch workspaces, and
// the batch launcher.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/lqg.h"
#include "lqg_internal.h"

namespace lqg_host {

using lqg::ExactScratch;
using lqg::SearchArgs;

lqg_status fail(lqg_status s, const std::string& msg);
lqg_status cuda_fail(cudaError_t e, const char* what);

#define LQG_CUDA(call)                                                \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return ::lqg_host::cuda_fail(e_, #call); \
    } while (0)

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// Control words in device memory, zeroed before every batch.
enum : int {
    kCtlFastHead = 0,
    kCtlFlagged = 1,
    kCtlExactHead = 2,
    kCtlErr = 3,
    kCtlErrQuery = 4,
    kCtlHeapHead = 5,
    kCtlSpilled = 6
};
constexpr int kCtlWords = 8;

constexpr uint32_t kMaxEf = 512;
constexpr uint32_t kHeapGlobalCap = 28672;  // heap kernel search-pool slots in global memory

// Mutable device state of one batch in flight: control words, the list of
// tie-flagged queries, the exact kernel's work areas, and staging buffers for
// the host-buffer entry points. Batches that overlap (on different streams)
// each need their own.
struct Workspace {
    uint32_t* d_ctl = nullptr;
    int32_t* d_flagged = nullptr;  // fast kernel -> heap kernel
    int32_t* d_spill = nullptr;    // heap/replay kernel -> exact kernel (2 x flagged_cap)
    int64_t flagged_cap = 0;
    ExactScratch xs{};
    uint2* d_sp_global = nullptr;  // heap kernel: search-pool slots beyond shared memory
    uint4* d_rlog = nullptr;       // replay kernel: per-query result logs
    uint32_t* d_rlen = nullptr;    // replay kernel: per-query log lengths
    size_t cap_rlog = 0, cap_rlen = 0;
    uint2* d_plog = nullptr;       // batch kernel, lazy heap: per-query pop logs
    size_t cap_plog = 0;
    uint32_t* d_okey = nullptr;    // work order: keys and query indices, in and out
    int32_t* d_oidx = nullptr;     //   (4 x chunk entries each)
    unsigned char* d_otemp = nullptr;  // work order: radix-sort scratch
    size_t cap_okey = 0, cap_oidx = 0, cap_otemp = 0;
    size_t sp_global_slots = 0;    // warps covered
    int x_blocks = 0, x_warps_per_block = 4;
    float* d_q = nullptr;
    uint32_t* d_kq = nullptr;
    uint32_t* d_efq = nullptr;
    uint32_t* d_ids = nullptr;
    uint32_t* d_pool_ids = nullptr;
    float* d_pool_d = nullptr;
    uint32_t* d_stats = nullptr;
    size_t cap_q = 0, cap_kq = 0, cap_efq = 0, cap_ids = 0, cap_pool_ids = 0, cap_pool_d = 0,
           cap_stats = 0;
    // one-query calls: pinned host staging for the query, the ids and the
    // control words, so the copies are plain DMA and one synchronisation ends
    // the call
    unsigned char* h_plain = nullptr;
    size_t cap_h_plain = 0;
    void release() {
        if (h_plain) cudaFreeHost(h_plain);
        h_plain = nullptr;
        cap_h_plain = 0;
        dfree(d_ctl);
        dfree(d_flagged);
        dfree(d_spill);
        flagged_cap = 0;
        dfree(xs.vis);
        dfree(xs.sp);
        dfree(xs.rp);
        dfree(d_sp_global);
        dfree(d_rlog);
        dfree(d_rlen);
        dfree(d_plog);
        cap_rlog = cap_rlen = cap_plog = 0;
        dfree(d_okey);
        dfree(d_oidx);
        dfree(d_otemp);
        cap_okey = cap_oidx = cap_otemp = 0;
        sp_global_slots = 0;
        dfree(d_q);
        dfree(d_kq);
        dfree(d_efq);
        dfree(d_ids);
        dfree(d_pool_ids);
        dfree(d_pool_d);
        dfree(d_stats);
        cap_q = cap_kq = cap_efq = cap_ids = cap_pool_ids = cap_pool_d = cap_stats = 0;
    }
};

// Makes ix->device current for the scope of a call.
struct DeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

struct BatchSpec {
    const float* q;
    int64_t m;
    const uint32_t* kq;
    uint32_t k0;
    const uint32_t* efq;
    uint32_t ef0;
    uint32_t* ids;
    uint32_t kstride;
    uint32_t* pool_ids;
    float* pool_d;
    uint32_t pstride;
    uint32_t* stats;
    cudaStream_t st;
    uint32_t ties_ok = 0;
    uint32_t* path = nullptr;  // index build: popped ids per query (fast kernel)
    uint32_t path_stride = 0;
    // the query-per-block form may run (modes 5-6, small batches): false when
    // other batches share the device, where its idle helper warps would cost
    // throughput
    bool small_ok = true;
};

template <typename T>
lqg_status grow(T*& p, size_t& cap, size_t need) {
    if (need <= cap) return LQG_OK;
    dfree(p);
    cap = 0;
    if (cudaMalloc(&p, need * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return fail(LQG_ERR_NOMEM, "staging allocation failed");
    }
    cap = need;
    return LQG_OK;
}

lqg_status ensure_ctl(Workspace& w, int64_t m);
lqg_status ensure_exact(Workspace& w, int blocks, int warps_per_block);
lqg_status reset_ctl(Workspace& w, cudaStream_t st);
lqg_status read_status(Workspace& w, cudaStream_t st);

// FastScan section of an index (fastscan.cu): per node, the RaBitQ codes and
// factors of its neighbours around the node, and the rotation's diagonal.
// Host copies in the file's layout (codes in upstream's FastScan blocks),
// device rows in the search kernel's.
struct FsSection {
    bool ready = false;
    uint32_t P = 0;                 // padded dimension
    std::vector<float> diag;        // [P]
    std::vector<uint8_t> packed;    // [n][deg * P / 8]
    std::vector<float> factors;     // [n][3][deg]
    unsigned char* d_rows = nullptr;
    float* d_diag = nullptr;
    uint64_t row_bytes = 0;
    uint32_t off_codes = 0, off_fac = 0, off_ids = 0;
    void release() {
        dfree(d_rows);
        dfree(d_diag);
        ready = false;
    }
};

}  // namespace lqg_host

struct lqg_index {
    uint64_t n = 0;
    uint32_t dim = 0, deg = 0, cstride = 0;
    int device = 0;
    uint32_t entry = 0;
    uint32_t ef = 0;  // 0 until lqg_set_ef (the reference leaves it undefined)
    bool has_data = false;
    int num_sms = 148;

    std::vector<float> vectors;   // [n][dim]
    std::vector<uint32_t> nbrs;   // [n][deg]
    std::vector<uint8_t> codes;   // [n][dim]
    std::vector<float> params;    // [dim][2]

    uint32_t* d_nbrs = nullptr;
    uint8_t* d_codes = nullptr;
    float* d_params = nullptr;

    lqg_host::Workspace ws;  // the default work area (one batch at a time)
    lqg_host::FsSection fs;  // FastScan section (empty until built or loaded)

    cudaStream_t own_stream = nullptr;
    // default: the batch kernel with the lazy search heap (mode 6), the
    // fastest on the bench batch and for single queries
    lqg_tuning tune{2, 10, 8, 0, 6, 4, 256, 15, 0, LQG_SMALL_BATCH_AUTO};
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;  // recorded around the fast kernel

    ~lqg_index() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        lqg_host::dfree(d_nbrs);
        lqg_host::dfree(d_codes);
        lqg_host::dfree(d_params);
        ws.release();
        fs.release();
        if (own_stream) cudaStreamDestroy(own_stream);
        cudaSetDevice(prev);
    }
};

namespace lqg_host {
lqg_status check_batch(lqg_index* ix, BatchSpec& b);
lqg_status run_batch(lqg_index* ix, Workspace& w, BatchSpec& b, bool plain);
// Work order of a batch (order.cu): largest ef, then farthest from the entry
// point, first.
lqg_status ensure_order(Workspace& w, int64_t chunk);
lqg_status order_queries(const lqg_index* ix, Workspace& w, const float* queries,
                         const uint32_t* efq, int64_t m, cudaStream_t st, const int32_t** list);
lqg_status search_host(lqg_index* ix, Workspace& w, const float* queries, int64_t m,
                       const uint32_t* k, uint32_t k0, const uint32_t* ef, uint32_t efb,
                       uint32_t* ids, uint32_t kstride, uint32_t* pool_ids, float* pool_d,
                       uint32_t pstride, uint32_t* stats, cudaStream_t st);
// FastScan section in the index file (fastscan.cu): appended after the
// reference's bytes, which the reference's loader reads and stops at.
uint64_t fs_file_bytes(const lqg_index* ix);
lqg_status fs_read(lqg_index* ix, FILE* f);
lqg_status fs_write(const lqg_index* ix, FILE* f);
}  // namespace lqg_host
