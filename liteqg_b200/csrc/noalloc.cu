// lqg_search_exact_noalloc: the exact search kernel with its work areas in a
// fixed array that is part of the library image, for callers that cannot let
// a library allocate GPU memory.
//
// Who needs it: applications whose GPU memory is already reserved by another
// allocator (for example a framework's caching pool that holds nearly all of
// the device), and latency-sensitive loops that must not call cudaMalloc or
// cudaFree, because those calls can synchronize the whole device and stall
// work on other streams. lqg_search_exact_device allocates its work areas on
// first use; this entry point never does.
//
// The array below is a per-device global of the library: every GPU that loads
// liblqg.so holds it until the process exits. Its size is fixed at build time
// (kNoAllocBytes, about 1.1 MB). It holds the control words (work-queue head,
// error word) and kNoAllocWarps per-warp work areas of the exact kernel:
// an exact visited set of 2^14 slots (at most 8192 visited nodes per query),
// a search heap of 8192 entries and a result heap of 520 entries (ef <= 512).
// A query that needs more fails with LQG_ERR_CAPACITY; its ids are LQG_NO_ID.
//
// All calls on a device share the one array and it keeps the last call's
// contents: each call zeroes the control words first, and the kernel clears a
// query's visited set before using it. Two calls whose work overlaps on the
// GPU (from different host threads or different streams) would race on the
// array, so such calls must be serialized by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "lqg_host.h"
#include "lqg_internal.h"

namespace {

constexpr int kNoAllocBlocks = 2;
constexpr int kNoAllocWarpsPerBlock = 4;
constexpr int kNoAllocWarps = kNoAllocBlocks * kNoAllocWarpsPerBlock;
constexpr uint32_t kNoAllocXBits = 14;
constexpr uint32_t kNoAllocSCap = 8192;
constexpr uint32_t kNoAllocRCap = lqg_host::kMaxEf + 8;
constexpr size_t kCtlBytes = 256;
constexpr size_t kVisBytes = (size_t)kNoAllocWarps * ((size_t)1 << kNoAllocXBits) * 4;
constexpr size_t kSpBytes = (size_t)kNoAllocWarps * kNoAllocSCap * 8;
constexpr size_t kRpBytes = (size_t)kNoAllocWarps * kNoAllocRCap * 8;
constexpr size_t kNoAllocBytes = kCtlBytes + kVisBytes + kSpBytes + kRpBytes;

// In host code this name only stands for the array; its device address comes
// from cudaGetSymbolAddress on each device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

static_assert(kNoAllocRCap >= lqg_host::kMaxEf + 2,
              "the result heap holds ef + 1 entries for every ef the host accepts");

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of the array on `device` (current). Looked up once per
// device, on the first call made on it, and kept for the life of the process:
// a device reset (cudaDeviceReset) after that first call is not supported,
// since the module is reloaded and the kept address goes stale.
lqg_status scratch_on(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices)
        return lqg_host::fail(LQG_ERR_ARG, "device ordinal out of range for the no-alloc entry");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return lqg_host::cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[device];
    return LQG_OK;
}

}  // namespace

extern "C" LQG_API lqg_status lqg_search_exact_noalloc(
    lqg_index* ix, const float* queries, int64_t m, const uint32_t* k, uint32_t k0,
    const uint32_t* ef, uint32_t ef0, uint32_t* ids, uint32_t kstride, uint32_t* pool_ids,
    float* pool_d, uint32_t pstride, uint32_t* stats, void* stream) {
    using namespace lqg_host;
    cudaStream_t st = (cudaStream_t)stream;
    BatchSpec b{queries, m, k, k0, ef, ef0, ids, kstride, pool_ids, pool_d, pstride, stats, st};
    lqg_status s = check_batch(ix, b);
    if (s != LQG_OK) return s;
    if (m == 0) return LQG_OK;
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    unsigned char* base = nullptr;
    if ((s = scratch_on(ix->device, &base)) != LQG_OK) return s;

    uint32_t* ctl = reinterpret_cast<uint32_t*>(base);
    ExactScratch xs{};
    xs.vis = reinterpret_cast<uint32_t*>(base + kCtlBytes);
    xs.sp = reinterpret_cast<uint2*>(base + kCtlBytes + kVisBytes);
    xs.rp = reinterpret_cast<uint2*>(base + kCtlBytes + kVisBytes + kSpBytes);
    xs.xbits = kNoAllocXBits;
    xs.scap = kNoAllocSCap;
    xs.rcap = kNoAllocRCap;

    // The array keeps the previous call's contents: reset the control words.
    LQG_CUDA(cudaMemsetAsync(ctl, 0, kCtlWords * sizeof(uint32_t), st));
    LQG_CUDA(cudaMemsetAsync(ctl + kCtlErrQuery, 0xFF, sizeof(uint32_t), st));

    SearchArgs x{};
    x.nbrs = ix->d_nbrs;
    x.codes = ix->d_codes;
    x.params = ix->d_params;
    x.n = (uint32_t)ix->n;
    x.dim = ix->dim;
    x.deg = ix->deg;
    x.cstride = ix->cstride;
    x.entry = ix->entry;
    x.queries = b.q;
    x.m = b.m;
    x.kq = b.kq;
    x.k0 = b.k0;
    x.efq = b.efq;
    x.ef0 = b.ef0;
    x.ids = b.ids;
    x.kstride = b.kstride;
    x.pool_ids = b.pool_ids;
    x.pool_d = b.pool_d;
    x.pstride = b.pstride;
    x.stats = b.stats;
    x.qhead = ctl + kCtlExactHead;
    x.err = ctl + kCtlErr;
    cudaError_t e = lqg::launch_exact(x, xs, (int)(ix->deg / 32), kNoAllocWarpsPerBlock,
                                      kNoAllocBlocks, st);
    if (e != cudaSuccess) return cuda_fail(e, "no-alloc exact search launch");

    // Report overflow of the fixed work areas: read the two error words.
    uint32_t err[2] = {0, 0};
    LQG_CUDA(cudaMemcpyAsync(err, ctl + kCtlErr, sizeof(err), cudaMemcpyDeviceToHost, st));
    LQG_CUDA(cudaStreamSynchronize(st));
    if (err[0])
        return fail(LQG_ERR_CAPACITY,
                    "query " + std::to_string(err[1]) +
                        " needs more than the no-alloc work area (8192 visited nodes, 8192 "
                        "search-heap entries)");
    return LQG_OK;
}
