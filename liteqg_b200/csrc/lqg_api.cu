// Host side of the B200 query path: the index object, the reference's file
// format, and the C ABI declared in include/lqg.h.
//
// Device layout of a loaded index (HBM, resident for the index's lifetime):
//   nbrs   [N][deg]      u32   neighbour ids, split out of the reference's
//                              float rows (symqglib/qg/qg.hpp:128-137, 420-436)
//   codes  [N][cstride]  u8    SQ8 codes, rows padded to a 16-byte multiple
//   params [D][2]        f32   (min, scale)
// The raw float vectors stay on the host: search never reads them
// (qg.hpp:325-328 reads only the codes), save() writes them back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lqg.h"
#include "lqg_build.h"
#include "lqg_host.h"
#include "lqg_internal.h"

namespace lqg_host {

namespace {
thread_local std::string g_last_error;
}  // namespace

lqg_status fail(lqg_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

lqg_status cuda_fail(cudaError_t e, const char* what) {
    return fail(LQG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

const char* last_error() { return g_last_error.c_str(); }

uint64_t file_bytes(uint64_t n, uint32_t dim, uint32_t deg) {
    return 4 + 4ull * n * (dim + deg) + n * (uint64_t)dim + 8ull * dim;
}

lqg_status validate_content(const lqg_index* ix) {
    if (ix->entry >= ix->n)
        return fail(LQG_ERR_CORRUPT, "entry point " + std::to_string(ix->entry) +
                                         " out of range (N=" + std::to_string(ix->n) + ")");
    const uint32_t* p = ix->nbrs.data();
    const uint64_t total = ix->n * ix->deg;
    for (uint64_t i = 0; i < total; ++i)
        if (p[i] >= ix->n)
            return fail(LQG_ERR_CORRUPT, "neighbour id " + std::to_string(p[i]) + " of node " +
                                             std::to_string(i / ix->deg) + " out of range");
    return LQG_OK;
}

lqg_status upload(lqg_index* ix) {
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    dfree(ix->d_nbrs);
    dfree(ix->d_codes);
    dfree(ix->d_params);
    const size_t nb = ix->n * ix->deg * sizeof(uint32_t);
    const size_t cb = ix->n * ix->cstride;
    if (cudaMalloc(&ix->d_nbrs, nb) != cudaSuccess || cudaMalloc(&ix->d_codes, cb) != cudaSuccess ||
        cudaMalloc(&ix->d_params, ix->dim * 2 * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        dfree(ix->d_nbrs);
        dfree(ix->d_codes);
        return fail(LQG_ERR_NOMEM, "device allocation of the index failed");
    }
    LQG_CUDA(cudaMemcpy(ix->d_nbrs, ix->nbrs.data(), nb, cudaMemcpyHostToDevice));
    if (ix->cstride != ix->dim) LQG_CUDA(cudaMemset(ix->d_codes, 0, cb));
    LQG_CUDA(cudaMemcpy2D(ix->d_codes, ix->cstride, ix->codes.data(), ix->dim, ix->dim, ix->n,
                          cudaMemcpyHostToDevice));
    LQG_CUDA(cudaMemcpy(ix->d_params, ix->params.data(), ix->dim * 2 * sizeof(float),
                        cudaMemcpyHostToDevice));
    ix->has_data = true;
    return LQG_OK;
}

int pool_regs_for(uint32_t ef_max) {
    int e = 1;
    while (32u * e < ef_max) e *= 2;
    return e;
}

lqg_status ensure_ctl(Workspace& w, int64_t m) {
    if (!w.d_ctl) {
        if (cudaMalloc(&w.d_ctl, kCtlWords * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            return fail(LQG_ERR_NOMEM, "control block allocation failed");
        }
    }
    if (w.flagged_cap < m) {
        dfree(w.d_flagged);
        dfree(w.d_spill);
        const int64_t cap = std::max<int64_t>(m, 1024);
        if (cudaMalloc(&w.d_flagged, cap * sizeof(int32_t)) != cudaSuccess ||
            cudaMalloc(&w.d_spill, 2 * cap * sizeof(int32_t)) != cudaSuccess) {
            cudaGetLastError();
            dfree(w.d_flagged);
            w.flagged_cap = 0;
            return fail(LQG_ERR_NOMEM, "flag list allocation failed");
        }
        w.flagged_cap = cap;
    }
    return LQG_OK;
}

// Exact-kernel work areas: blocks x warps_per_block warps, each with an exact
// visited set of 2^16 slots (up to 32768 visited nodes per query), a search
// heap of 32768 entries and a result heap of kMaxEf + 8 entries (about
// 0.5 MB per warp).
lqg_status ensure_exact(Workspace& w, int blocks, int warps_per_block) {
    if (w.xs.vis) return LQG_OK;
    w.x_blocks = blocks;
    w.x_warps_per_block = warps_per_block;
    w.xs.xbits = 16;
    w.xs.scap = 32768;
    w.xs.rcap = kMaxEf + 8;
    const size_t nw = (size_t)blocks * warps_per_block;
    if (cudaMalloc(&w.xs.vis, nw * ((size_t)1 << w.xs.xbits) * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&w.xs.sp, nw * w.xs.scap * sizeof(uint2)) != cudaSuccess ||
        cudaMalloc(&w.xs.rp, nw * w.xs.rcap * sizeof(uint2)) != cudaSuccess) {
        cudaGetLastError();
        dfree(w.xs.vis);
        dfree(w.xs.sp);
        dfree(w.xs.rp);
        return fail(LQG_ERR_NOMEM, "exact-kernel work area allocation failed");
    }
    return LQG_OK;
}

lqg_status check_batch(lqg_index* ix, BatchSpec& b) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (!ix->has_data) return fail(LQG_ERR_STATE, "index has no data: load or build it first");
    if (b.m < 0 || b.m > (int64_t)INT32_MAX) return fail(LQG_ERR_ARG, "bad query count");
    if (b.m > 0 && (!b.q || !b.ids)) return fail(LQG_ERR_ARG, "null queries or ids");
    if (!b.kq && b.k0 > b.kstride) return fail(LQG_ERR_ARG, "k exceeds kstride");
    if (b.kstride == 0) return fail(LQG_ERR_ARG, "kstride must be > 0");
    if (!b.efq && b.ef0 == 0) {
        if (ix->ef == 0) return fail(LQG_ERR_STATE, "ef not set: call set_ef first");
        b.ef0 = ix->ef;
    }
    if (b.ef0 == 0 || b.ef0 > kMaxEf)
        return fail(LQG_ERR_ARG, "ef (or the per-query ef bound) must be in [1, 512]");
    if ((b.pool_ids == nullptr) != (b.pool_d == nullptr))
        return fail(LQG_ERR_ARG, "pool_ids and pool_d go together");
    if (b.pool_ids && b.pstride == 0) return fail(LQG_ERR_ARG, "pstride must be > 0");
    return LQG_OK;
}

SearchArgs base_args(const lqg_index* ix, const Workspace& w, const BatchSpec& b) {
    SearchArgs a{};
    a.nbrs = ix->d_nbrs;
    a.codes = ix->d_codes;
    a.params = ix->d_params;
    a.n = (uint32_t)ix->n;
    a.dim = ix->dim;
    a.deg = ix->deg;
    a.cstride = ix->cstride;
    a.entry = ix->entry;
    a.queries = b.q;
    a.m = b.m;
    a.kq = b.kq;
    a.k0 = b.k0;
    a.efq = b.efq;
    a.ef0 = b.ef0;
    a.ids = b.ids;
    a.kstride = b.kstride;
    a.pool_ids = b.pool_ids;
    a.pool_d = b.pool_d;
    a.pstride = b.pstride;
    a.stats = b.stats;
    a.err = w.d_ctl + kCtlErr;
    return a;
}

lqg_status reset_ctl(Workspace& w, cudaStream_t st) {
    LQG_CUDA(cudaMemsetAsync(w.d_ctl, 0, kCtlWords * sizeof(uint32_t), st));
    LQG_CUDA(cudaMemsetAsync(w.d_ctl + kCtlErrQuery, 0xFF, sizeof(uint32_t), st));
    return LQG_OK;
}

// Fast kernel over all queries, then the exact kernel over the flagged ones.
// `plain` launches one warp (the one-query-per-launch form).
lqg_status run_batch(lqg_index* ix, Workspace& w, BatchSpec& b, bool plain) {
    lqg_status s = check_batch(ix, b);
    if (s != LQG_OK) return s;
    if (b.m == 0) return LQG_OK;
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    if ((s = ensure_ctl(w, b.m)) != LQG_OK) return s;
    if ((s = ensure_exact(w, ix->num_sms, 4)) != LQG_OK) return s;
    if ((s = reset_ctl(w, b.st)) != LQG_OK) return s;

    const int E = pool_regs_for(b.ef0);
    const int degw = (int)(ix->deg / 32);
    const lqg_tuning& t = ix->tune;
    const bool heap_all = t.mode == 2;
    cudaError_t e;

    if (t.mode >= 3) {
        // replay (3), split (4) or batch (5; 6 with the lazy search heap)
        // kernel over every query, then the result replay pass where the
        // search warps do not replay in place, in chunks whose logs fit
        // 1.5 GiB; spilled queries go to the exact kernel
        const bool lazy = t.mode == 6;
        const bool batch = t.mode == 5 || lazy;
        const bool split = t.mode == 4 || batch;
        const int RE = lqg::replay_pool_regs(b.ef0);
        if (RE == 0) return fail(LQG_ERR_ARG, "ef too large for the replay kernels");
        lqg::ReplayArgs ra{};
        ra.rcap = (b.ef0 + 2u) & ~1u;
        ra.efcap = std::min(32u * (uint32_t)RE - 32u, ra.rcap - 1u);
        ra.scap = t.heap_scap;
        ra.spill = w.d_spill;
        ra.nspill = w.d_ctl + kCtlSpilled;
        ra.rlog_cap = std::max(1024u, 16u * b.ef0);
        ra.replay_all = t.replay_all;
        ra.acap = 32u * (uint32_t)RE;
        ra.lazy = lazy ? 1u : 0u;
        const int64_t chunk = std::min<int64_t>(
            b.m, std::max<int64_t>(1024, (int64_t(1) << 30) / ((int64_t)ra.rlog_cap * 16)));
        if ((s = grow(w.d_rlog, w.cap_rlog, (size_t)chunk * ra.rlog_cap)) != LQG_OK) return s;
        if ((s = grow(w.d_rlen, w.cap_rlen, (size_t)chunk)) != LQG_OK) return s;
        if (lazy && (s = grow(w.d_plog, w.cap_plog, (size_t)chunk * ra.rlog_cap)) != LQG_OK)
            return s;
        ra.plog = lazy ? w.d_plog : nullptr;
        ra.rlog = w.d_rlog;
        ra.rlen = w.d_rlen;
        // split kernel blocks hold at most 5 warps (its 96-register budget)
        int sw = plain ? 1 : (int)(split ? std::min(t.heap_warps, 5u) : t.replay_warps);
        if (batch) {
            while (sw > 1 &&
                   lqg::batch_smem_bytes(ix->dim, t.visited_bits, ra.scap, ra.acap, sw) > 227 * 1024)
                --sw;
        } else if (split) {
            while (sw > 1 && lqg::split_smem_bytes(ix->dim, t.visited_bits, ra.scap, sw) > 227 * 1024)
                --sw;
        } else {
            while (sw > 1 && lqg::replay_smem_bytes(ix->dim, t.visited_bits, ra.scap, sw) > 227 * 1024)
                --sw;
        }
        ra.swarps = (uint32_t)sw;
        SearchArgs h = base_args(ix, w, b);
        h.qhead = w.d_ctl + kCtlHeapHead;
        h.vbits = t.visited_bits;
        // small batches: one query per block of 4 warps, when every query of
        // the batch can be resident at once
        bool cta = false;
        if (batch && b.small_ok && t.small_batch != LQG_SMALL_BATCH_OFF &&
            lqg::batch_smem_bytes(ix->dim, t.visited_bits, ra.scap, ra.acap, 1) <= 227 * 1024) {
            if (plain) {
                cta = true;  // one query: no occupancy question
            } else {
                int oc = 0;
                e = lqg::launch_batch_cta(h, ra, degw, 0, b.st, &oc);
                if (e != cudaSuccess) return cuda_fail(e, "small-batch kernel occupancy");
                const int64_t lim = t.small_batch == LQG_SMALL_BATCH_AUTO
                                        ? (int64_t)oc * ix->num_sms
                                        : t.small_batch;
                cta = oc > 0 && b.m <= lim;
            }
        }
        if (cta) sw = 1;
        auto launch = [&](const SearchArgs& c, int blocks, int* occ) {
            if (cta) return lqg::launch_batch_cta(c, ra, degw, blocks, b.st, occ);
            if (batch)
                return lqg::launch_batch(c, ra, (int)t.lanes_per_cand, degw, sw, blocks, b.st, occ);
            return split ? lqg::launch_split(c, ra, RE, (int)t.lanes_per_cand, degw, sw, blocks, b.st, occ)
                         : lqg::launch_replay(c, ra, RE, (int)t.lanes_per_cand, degw, blocks, b.st, occ);
        };
        int rb = 1;
        if (!plain) {
            int occ = 0;
            e = launch(h, 0, &occ);
            if (e != cudaSuccess || occ <= 0)
                return fail(LQG_ERR_ARG, "search kernel cannot launch with this tuning");
            rb = occ * ix->num_sms;
            const int64_t need = (chunk + sw - 1) / sw;
            if (need < rb) rb = (int)need;
        }
        // longest-expected queries first, when a chunk holds more queries
        // than the launch has warps (otherwise they all start at once)
        const bool order = !plain && chunk > (int64_t)rb * sw;
        if (order && (s = ensure_order(w, chunk)) != LQG_OK) return s;
        const size_t slots = (size_t)rb * sw;
        if (w.sp_global_slots < slots) {
            dfree(w.d_sp_global);
            w.sp_global_slots = 0;
            if (cudaMalloc(&w.d_sp_global, slots * kHeapGlobalCap * sizeof(uint2)) != cudaSuccess) {
                cudaGetLastError();
                return fail(LQG_ERR_NOMEM, "search-pool area allocation failed");
            }
            w.sp_global_slots = slots;
        }
        ra.sp_global = w.d_sp_global;
        ra.gcap = kHeapGlobalCap;
        if (ix->ev_start) LQG_CUDA(cudaEventRecord(ix->ev_start, b.st));
        for (int64_t off = 0; off < b.m; off += chunk) {
            const int64_t mc = std::min(chunk, b.m - off);
            if (off > 0) {  // fresh work-queue heads and spill list for this chunk
                LQG_CUDA(cudaMemsetAsync(w.d_ctl + kCtlExactHead, 0, sizeof(uint32_t), b.st));
                LQG_CUDA(cudaMemsetAsync(w.d_ctl + kCtlHeapHead, 0, 2 * sizeof(uint32_t), b.st));
            }
            SearchArgs c = h;
            c.queries += off * ix->dim;
            if (c.kq) c.kq += off;
            if (c.efq) c.efq += off;
            c.ids += off * b.kstride;
            if (c.pool_ids) {
                c.pool_ids += off * b.pstride;
                c.pool_d += off * b.pstride;
            }
            if (c.stats) c.stats += off * 4;
            c.m = mc;
            if (order && mc > (int64_t)rb * sw &&
                (s = order_queries(ix, w, c.queries, c.efq, mc, b.st, &c.qlist)) != LQG_OK)
                return s;
            const int cb = (int)std::min<int64_t>(rb, (mc + sw - 1) / sw);
            e = launch(c, cb, nullptr);
            if (e != cudaSuccess) return cuda_fail(e, "search launch");
            const bool in_place =
                batch ? lqg::batch_replays_in_place_host(t.visited_bits, ra.scap, ra.acap, ra.rcap)
                      : lqg::split_replays_in_place_host(t.visited_bits, ra.scap, ra.rcap);
            if (!split || ra.replay_all || !in_place) {
                e = lqg::launch_rp_replay(c, ra, b.st);
                if (e != cudaSuccess) return cuda_fail(e, "result replay launch");
            }
            SearchArgs x = c;
            x.qlist = w.d_spill;
            x.nlist = w.d_ctl + kCtlSpilled;
            x.qhead = w.d_ctl + kCtlExactHead;
            e = lqg::launch_exact(x, w.xs, degw, plain ? 1 : w.x_warps_per_block,
                                  plain ? 1 : w.x_blocks, b.st);
            if (e != cudaSuccess) return cuda_fail(e, "exact search launch");
        }
        if (ix->ev_stop) LQG_CUDA(cudaEventRecord(ix->ev_stop, b.st));
        return LQG_OK;
    } else {

    // work order of the batch: longest-expected queries first
    const int32_t* order = nullptr;
    // (only when the batch is larger than about one wave of resident warps;
    // smaller batches start all their queries at once)
    if (!plain && b.m > (int64_t)ix->num_sms * 16) {
        if ((s = ensure_order(w, b.m)) != LQG_OK) return s;
        if ((s = order_queries(ix, w, b.q, b.efq, b.m, b.st, &order)) != LQG_OK) return s;
    }

    // 1. fast kernel over every query (mode 1); tied queries go to the list
    if (!heap_all) {
        SearchArgs a = base_args(ix, w, b);
        a.qhead = w.d_ctl + kCtlFastHead;
        a.nflagged = w.d_ctl + kCtlFlagged;
        a.flagged = w.d_flagged;
        a.vbits = t.visited_bits;
        a.ties_ok = b.ties_ok;
        a.path = b.path;
        a.path_stride = b.path_stride;
        a.qlist = order;
        int warps = plain ? 1 : (int)t.warps_per_block;
        int blocks = 1;
        if (!plain) {
            int occ = t.blocks_per_sm ? (int)t.blocks_per_sm
                                      : lqg::fast_occupancy(E, (int)t.lanes_per_cand, degw, warps,
                                                            ix->dim, t.visited_bits);
            if (occ <= 0) return fail(LQG_ERR_ARG, "fast kernel cannot launch with this tuning");
            blocks = occ * ix->num_sms;
            const int64_t need = (b.m + warps - 1) / warps;
            if (need < blocks) blocks = (int)need;
        }
        if (ix->ev_start) LQG_CUDA(cudaEventRecord(ix->ev_start, b.st));
        e = lqg::launch_fast(a, E, (int)t.lanes_per_cand, degw, warps, blocks, b.st);
        if (e != cudaSuccess) return cuda_fail(e, "fast search launch");
    }

    // 2. heap kernel: the flagged queries (mode 1) or all of them (mode 2)
    {
        SearchArgs h = base_args(ix, w, b);
        if (!heap_all) {
            h.qlist = w.d_flagged;
            h.nlist = w.d_ctl + kCtlFlagged;
        } else {
            h.qlist = order;
        }
        h.qhead = w.d_ctl + kCtlHeapHead;
        h.vbits = t.visited_bits;
        lqg::HeapArgs hp{};
        hp.rcap = (b.ef0 + 2u) & ~1u;
        hp.scap = t.heap_scap;
        hp.spill = w.d_spill;
        hp.nspill = w.d_ctl + kCtlSpilled;
        int hw = plain ? 1 : (int)t.heap_warps;
        int hb = 1;
        if (!plain) {
            int occ = 0;
            e = lqg::launch_heap(h, hp, (int)t.lanes_per_cand, degw, hw, 0, b.st, &occ);
            if (e != cudaSuccess || occ <= 0)
                return fail(LQG_ERR_ARG, "heap kernel cannot launch with this tuning");
            hb = occ * ix->num_sms;
            const int64_t need = (b.m + hw - 1) / hw;
            if (need < hb) hb = (int)need;
        }
        const size_t slots = (size_t)hb * hw;
        if (w.sp_global_slots < slots) {
            dfree(w.d_sp_global);
            w.sp_global_slots = 0;
            if (cudaMalloc(&w.d_sp_global, slots * kHeapGlobalCap * sizeof(uint2)) != cudaSuccess) {
                cudaGetLastError();
                return fail(LQG_ERR_NOMEM, "heap kernel search-pool area allocation failed");
            }
            w.sp_global_slots = slots;
        }
        hp.sp_global = w.d_sp_global;
        hp.gcap = kHeapGlobalCap;
        if (heap_all && ix->ev_start) LQG_CUDA(cudaEventRecord(ix->ev_start, b.st));
        e = lqg::launch_heap(h, hp, (int)t.lanes_per_cand, degw, hw, hb, b.st, nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "heap search launch");
    }
    }

    // 3. exact global-memory kernel: queries whose search pool outgrew shared memory
    SearchArgs x = base_args(ix, w, b);
    x.qlist = w.d_spill;
    x.nlist = w.d_ctl + kCtlSpilled;
    x.qhead = w.d_ctl + kCtlExactHead;
    int xb = plain ? 1 : w.x_blocks;
    int xw = plain ? 1 : w.x_warps_per_block;
    e = lqg::launch_exact(x, w.xs, degw, xw, xb, b.st);
    if (e != cudaSuccess) return cuda_fail(e, "exact search launch");
    if (ix->ev_stop) LQG_CUDA(cudaEventRecord(ix->ev_stop, b.st));
    return LQG_OK;
}

// The status of a finished batch from its control words.
lqg_status status_of(const uint32_t* ctl) {
    if (ctl[kCtlErr]) {
        std::string why;
        if (ctl[kCtlErr] & lqg::kErrVisitedFull) why += " visited set full (32768 nodes);";
        if (ctl[kCtlErr] & lqg::kErrHeapFull) why += " search heap full (32768 entries);";
        if (ctl[kCtlErr] & lqg::kErrProbe) why += " visited-set probe failed;";
        if (ctl[kCtlErr] & lqg::kErrSync)
            return fail(LQG_ERR_CUDA, "replay kernel: a wait between its warps timed out");
        return fail(LQG_ERR_CAPACITY, "exact search work area overflow for query " +
                                          std::to_string(ctl[kCtlErrQuery]) + ":" + why);
    }
    return LQG_OK;
}

lqg_status read_status(Workspace& w, cudaStream_t st) {
    uint32_t ctl[kCtlWords];
    LQG_CUDA(cudaMemcpyAsync(ctl, w.d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st));
    LQG_CUDA(cudaStreamSynchronize(st));
    return status_of(ctl);
}

// Host-buffer batch: copy in, search, copy out, wait (one workspace).
lqg_status search_host(lqg_index* ix, Workspace& w, const float* queries, int64_t m,
                       const uint32_t* k, uint32_t k0, const uint32_t* ef, uint32_t efb,
                       uint32_t* ids, uint32_t kstride, uint32_t* pool_ids, float* pool_d,
                       uint32_t pstride, uint32_t* stats, cudaStream_t st) {
    lqg_status s;
    if ((s = grow(w.d_q, w.cap_q, (size_t)m * ix->dim)) != LQG_OK) return s;
    if ((s = grow(w.d_ids, w.cap_ids, (size_t)m * kstride)) != LQG_OK) return s;
    if (k && (s = grow(w.d_kq, w.cap_kq, (size_t)m)) != LQG_OK) return s;
    if (ef && (s = grow(w.d_efq, w.cap_efq, (size_t)m)) != LQG_OK) return s;
    if (stats && (s = grow(w.d_stats, w.cap_stats, (size_t)m * 4)) != LQG_OK) return s;
    if (pool_ids) {
        if ((s = grow(w.d_pool_ids, w.cap_pool_ids, (size_t)m * pstride)) != LQG_OK) return s;
        if ((s = grow(w.d_pool_d, w.cap_pool_d, (size_t)m * pstride)) != LQG_OK) return s;
    }
    LQG_CUDA(cudaMemcpyAsync(w.d_q, queries, (size_t)m * ix->dim * 4, cudaMemcpyHostToDevice, st));
    if (k) LQG_CUDA(cudaMemcpyAsync(w.d_kq, k, m * 4, cudaMemcpyHostToDevice, st));
    if (ef) LQG_CUDA(cudaMemcpyAsync(w.d_efq, ef, m * 4, cudaMemcpyHostToDevice, st));
    BatchSpec b{w.d_q,
                m,
                k ? w.d_kq : nullptr,
                k0,
                ef ? w.d_efq : nullptr,
                efb,
                w.d_ids,
                kstride,
                pool_ids ? w.d_pool_ids : nullptr,
                pool_ids ? w.d_pool_d : nullptr,
                pstride,
                stats ? w.d_stats : nullptr,
                st};
    if ((s = run_batch(ix, w, b, false)) != LQG_OK) return s;
    LQG_CUDA(cudaMemcpyAsync(ids, w.d_ids, (size_t)m * kstride * 4, cudaMemcpyDeviceToHost, st));
    if (pool_ids) {
        LQG_CUDA(cudaMemcpyAsync(pool_ids, w.d_pool_ids, (size_t)m * pstride * 4,
                                 cudaMemcpyDeviceToHost, st));
        LQG_CUDA(cudaMemcpyAsync(pool_d, w.d_pool_d, (size_t)m * pstride * 4,
                                 cudaMemcpyDeviceToHost, st));
    }
    if (stats)
        LQG_CUDA(cudaMemcpyAsync(stats, w.d_stats, (size_t)m * 16, cudaMemcpyDeviceToHost, st));
    return read_status(w, st);
}

}  // namespace lqg_host

using namespace lqg_host;

extern "C" {

const char* lqg_last_error(void) { return lqg_host::last_error(); }

lqg_status lqg_create(const char* index_type, const char* metric, uint64_t num_elements,
                      uint32_t dimension, uint32_t degree_bound, int device, lqg_index** out) {
    if (!out) return fail(LQG_ERR_ARG, "null output handle");
    *out = nullptr;
    if (!metric || std::string(metric) != "L2")
        return fail(LQG_ERR_ARG, "Only L2 distance supported currently");
    if (degree_bound < 32 || degree_bound % 32 != 0)
        return fail(LQG_ERR_ARG, "The degree bound must be a multiple of 32");
    if (!index_type || std::string(index_type) != "QG")
        return fail(LQG_ERR_ARG, std::string("Index type [") + (index_type ? index_type : "") +
                                     "] not supported");
    if (degree_bound > lqg::kMaxDeg)
        return fail(LQG_ERR_ARG, "degree_bound above 128 is not supported on the GPU");
    if (dimension < 33 || dimension > 2048)
        return fail(LQG_ERR_ARG, "dimension must be in [33, 2048]");
    if (num_elements == 0 || num_elements >= (1ull << 31))
        return fail(LQG_ERR_ARG, "num_elements must be in [1, 2^31)");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) return fail(LQG_ERR_ARG, "bad device ordinal");
    auto* ix = new (std::nothrow) lqg_index();
    if (!ix) return fail(LQG_ERR_NOMEM, "host allocation failed");
    ix->n = num_elements;
    ix->dim = dimension;
    ix->deg = degree_bound;
    ix->cstride = (dimension + 15u) & ~15u;
    ix->device = device;
    cudaDeviceGetAttribute(&ix->num_sms, cudaDevAttrMultiProcessorCount, device);
    *out = ix;
    return LQG_OK;
}

void lqg_free(lqg_index* ix) { delete ix; }

lqg_status lqg_load(lqg_index* ix, const char* path) {
    if (!ix || !path) return fail(LQG_ERR_ARG, "null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(LQG_ERR_IO, std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    const long long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    const uint64_t want = file_bytes(ix->n, ix->dim, ix->deg);
    // the reference's bytes, optionally followed by a FastScan section
    const bool with_fs = size >= 0 && (uint64_t)size == want + fs_file_bytes(ix);
    if (size < 0 || ((uint64_t)size != want && !with_fs)) {
        std::fclose(f);
        return fail(LQG_ERR_IO, std::string(path) + ": " + std::to_string(size) +
                                    " bytes, expected " + std::to_string(want) +
                                    " for the index's N, dimension and degree_bound");
    }
    ix->fs.release();
    try {
        ix->vectors.resize(ix->n * ix->dim);
        ix->nbrs.resize(ix->n * ix->deg);
        ix->codes.resize(ix->n * ix->dim);
        ix->params.resize(ix->dim * 2);
    } catch (...) {
        std::fclose(f);
        return fail(LQG_ERR_NOMEM, "host allocation failed");
    }
    bool ok = std::fread(&ix->entry, 4, 1, f) == 1;
    const size_t row = ix->dim + ix->deg;
    std::vector<uint32_t> buf;
    const size_t chunk = 1 << 16;
    for (uint64_t i0 = 0; ok && i0 < ix->n; i0 += chunk) {
        const size_t rows = std::min<uint64_t>(chunk, ix->n - i0);
        buf.resize(rows * row);
        ok = std::fread(buf.data(), 4, rows * row, f) == rows * row;
        for (size_t r = 0; ok && r < rows; ++r) {
            std::memcpy(&ix->vectors[(i0 + r) * ix->dim], &buf[r * row], 4 * ix->dim);
            std::memcpy(&ix->nbrs[(i0 + r) * ix->deg], &buf[r * row + ix->dim], 4 * ix->deg);
        }
    }
    ok = ok && std::fread(ix->codes.data(), 1, ix->codes.size(), f) == ix->codes.size();
    ok = ok && std::fread(ix->params.data(), 4, ix->params.size(), f) == ix->params.size();
    if (!ok) {
        std::fclose(f);
        return fail(LQG_ERR_IO, std::string("short read from ") + path);
    }
    lqg_status s = validate_content(ix);
    if (s == LQG_OK) s = upload(ix);
    if (s == LQG_OK && with_fs) s = fs_read(ix, f);
    std::fclose(f);
    return s;
}

lqg_status lqg_save(const lqg_index* ix, const char* path) {
    if (!ix || !path) return fail(LQG_ERR_ARG, "null argument");
    if (!ix->has_data) return fail(LQG_ERR_STATE, "index has no data");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(LQG_ERR_IO, std::string("cannot create ") + path);
    bool ok = std::fwrite(&ix->entry, 4, 1, f) == 1;
    const size_t row = ix->dim + ix->deg;
    std::vector<uint32_t> buf;
    const size_t chunk = 1 << 16;
    for (uint64_t i0 = 0; ok && i0 < ix->n; i0 += chunk) {
        const size_t rows = std::min<uint64_t>(chunk, ix->n - i0);
        buf.resize(rows * row);
        for (size_t r = 0; r < rows; ++r) {
            std::memcpy(&buf[r * row], &ix->vectors[(i0 + r) * ix->dim], 4 * ix->dim);
            std::memcpy(&buf[r * row + ix->dim], &ix->nbrs[(i0 + r) * ix->deg], 4 * ix->deg);
        }
        ok = std::fwrite(buf.data(), 4, rows * row, f) == rows * row;
    }
    ok = ok && std::fwrite(ix->codes.data(), 1, ix->codes.size(), f) == ix->codes.size();
    ok = ok && std::fwrite(ix->params.data(), 4, ix->params.size(), f) == ix->params.size();
    if (ok && ix->fs.ready) ok = fs_write(ix, f) == LQG_OK;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? LQG_OK : fail(LQG_ERR_IO, std::string("write to ") + path + " failed");
}

lqg_status lqg_set_arrays(lqg_index* ix, uint32_t entry, const float* vectors,
                          const uint32_t* nbrs, const uint8_t* codes, const float* params) {
    if (!ix || !nbrs || !codes || !params) return fail(LQG_ERR_ARG, "null argument");
    try {
        ix->vectors.assign(ix->n * ix->dim, 0.f);
        if (vectors) std::memcpy(ix->vectors.data(), vectors, ix->vectors.size() * 4);
        ix->nbrs.assign(nbrs, nbrs + ix->n * ix->deg);
        ix->codes.assign(codes, codes + ix->n * ix->dim);
        ix->params.assign(params, params + ix->dim * 2);
    } catch (...) {
        return fail(LQG_ERR_NOMEM, "host allocation failed");
    }
    ix->entry = entry;
    ix->fs.release();  // the graph changed: its FastScan section is stale
    lqg_status s = validate_content(ix);
    if (s != LQG_OK) return s;
    return upload(ix);
}

lqg_status lqg_get_arrays(const lqg_index* ix, uint32_t* entry, float* vectors, uint32_t* nbrs,
                          uint8_t* codes, float* params) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (!ix->has_data) return fail(LQG_ERR_STATE, "index has no data");
    if (entry) *entry = ix->entry;
    if (vectors) std::memcpy(vectors, ix->vectors.data(), ix->vectors.size() * 4);
    if (nbrs) std::memcpy(nbrs, ix->nbrs.data(), ix->nbrs.size() * 4);
    if (codes) std::memcpy(codes, ix->codes.data(), ix->codes.size());
    if (params) std::memcpy(params, ix->params.data(), ix->params.size() * 4);
    return LQG_OK;
}

lqg_status lqg_set_ef(lqg_index* ix, uint32_t ef) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (ef == 0 || ef > kMaxEf) return fail(LQG_ERR_ARG, "ef must be in [1, 512]");
    ix->ef = ef;
    return LQG_OK;
}

lqg_status lqg_search(lqg_index* ix, const float* query, uint32_t k, uint32_t* results) {
    if (!ix || !query || !results) return fail(LQG_ERR_ARG, "null argument");
    if (k == 0) return LQG_OK;
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    if (!ix->own_stream) LQG_CUDA(cudaStreamCreateWithFlags(&ix->own_stream, cudaStreamNonBlocking));
    lqg_status s;
    Workspace& w = ix->ws;
    if ((s = grow(w.d_q, w.cap_q, ix->dim)) != LQG_OK) return s;
    if ((s = grow(w.d_ids, w.cap_ids, k)) != LQG_OK) return s;
    cudaStream_t st = ix->own_stream;
    // pinned staging: query | ids | control words, each on 16 bytes
    const size_t qb = ((size_t)ix->dim * 4 + 15) & ~(size_t)15;
    const size_t ib = ((size_t)k * 4 + 15) & ~(size_t)15;
    const size_t need = qb + ib + kCtlWords * sizeof(uint32_t);
    if (w.cap_h_plain < need) {
        if (w.h_plain) cudaFreeHost(w.h_plain);
        w.h_plain = nullptr;
        w.cap_h_plain = 0;
        if (cudaHostAlloc(&w.h_plain, need, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return fail(LQG_ERR_NOMEM, "pinned staging allocation failed");
        }
        w.cap_h_plain = need;
    }
    float* h_q = reinterpret_cast<float*>(w.h_plain);
    uint32_t* h_ids = reinterpret_cast<uint32_t*>(w.h_plain + qb);
    uint32_t* h_ctl = reinterpret_cast<uint32_t*>(w.h_plain + qb + ib);
    std::memcpy(h_q, query, (size_t)ix->dim * 4);
    LQG_CUDA(cudaMemcpyAsync(w.d_q, h_q, ix->dim * 4, cudaMemcpyHostToDevice, st));
    BatchSpec b{w.d_q, 1, nullptr, k, nullptr, 0, w.d_ids, k, nullptr, nullptr, 0, nullptr, st};
    if ((s = run_batch(ix, w, b, true)) != LQG_OK) return s;
    LQG_CUDA(cudaMemcpyAsync(h_ids, w.d_ids, k * 4, cudaMemcpyDeviceToHost, st));
    LQG_CUDA(cudaMemcpyAsync(h_ctl, w.d_ctl, kCtlWords * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             st));
    LQG_CUDA(cudaStreamSynchronize(st));
    std::memcpy(results, h_ids, (size_t)k * 4);
    return status_of(h_ctl);
}

lqg_status lqg_search_batch_device(lqg_index* ix, const float* queries, int64_t m,
                                   const uint32_t* k, uint32_t k0, const uint32_t* ef,
                                   uint32_t ef0, uint32_t* ids, uint32_t kstride,
                                   uint32_t* pool_ids, float* pool_d, uint32_t pstride,
                                   uint32_t* stats, void* stream) {
    BatchSpec b{queries, m,      k,      k0,      ef,    ef0,   ids,
                kstride, pool_ids, pool_d, pstride, stats, (cudaStream_t)stream};
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    return run_batch(ix, ix->ws, b, false);
}

lqg_status lqg_stream_status(lqg_index* ix, void* stream) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (!ix->ws.d_ctl) return LQG_OK;
    DeviceScope ds(ix->device);
    return read_status(ix->ws, (cudaStream_t)stream);
}

lqg_status lqg_search_batch(lqg_index* ix, const float* queries, int64_t m, const uint32_t* k,
                            uint32_t k0, const uint32_t* ef, uint32_t ef0, uint32_t* ids,
                            uint32_t kstride, uint32_t* pool_ids, float* pool_d,
                            uint32_t pstride, uint32_t* stats, void* stream) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (m <= 0) return m == 0 ? LQG_OK : fail(LQG_ERR_ARG, "bad query count");
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t efb = ef0;
    if (ef) {
        efb = 0;
        for (int64_t i = 0; i < m; ++i) efb = std::max(efb, ef[i]);
    }
    if (k)
        for (int64_t i = 0; i < m; ++i)
            if (k[i] > kstride) return fail(LQG_ERR_ARG, "k exceeds kstride");
    return search_host(ix, ix->ws, queries, m, k, k0, ef, efb, ids, kstride, pool_ids, pool_d,
                       pstride, stats, st);
}

lqg_status lqg_search_exact_device(lqg_index* ix, const float* queries, int64_t m,
                                   const uint32_t* k, uint32_t k0, const uint32_t* ef,
                                   uint32_t ef0, uint32_t* ids, uint32_t kstride,
                                   uint32_t* pool_ids, float* pool_d, uint32_t pstride,
                                   uint32_t* stats, void* stream) {
    BatchSpec b{queries, m,      k,      k0,      ef,    ef0,   ids,
                kstride, pool_ids, pool_d, pstride, stats, (cudaStream_t)stream};
    lqg_status s = check_batch(ix, b);
    if (s != LQG_OK) return s;
    if (m == 0) return LQG_OK;
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    Workspace& w = ix->ws;
    if ((s = ensure_ctl(w, 1)) != LQG_OK) return s;
    if ((s = ensure_exact(w, ix->num_sms, 4)) != LQG_OK) return s;
    if ((s = reset_ctl(w, b.st)) != LQG_OK) return s;
    SearchArgs x = base_args(ix, w, b);
    x.qhead = w.d_ctl + kCtlExactHead;
    cudaError_t e = lqg::launch_exact(x, w.xs, (int)(ix->deg / 32), w.x_warps_per_block,
                                      w.x_blocks, b.st);
    if (e != cudaSuccess) return cuda_fail(e, "exact search launch");
    return LQG_OK;
}

lqg_status lqg_set_kernel_events(lqg_index* ix, void* start, void* stop) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if ((start == nullptr) != (stop == nullptr)) return fail(LQG_ERR_ARG, "give both events or none");
    ix->ev_start = (cudaEvent_t)start;
    ix->ev_stop = (cudaEvent_t)stop;
    return LQG_OK;
}

lqg_status lqg_set_tuning(lqg_index* ix, const lqg_tuning* t) {
    if (!ix || !t) return fail(LQG_ERR_ARG, "null argument");
    lqg_tuning n = ix->tune;
    if (t->lanes_per_cand) {
        const uint32_t g = t->lanes_per_cand;
        if (g != 1 && g != 2 && g != 4 && g != 8 && g != 16)
            return fail(LQG_ERR_ARG, "lanes_per_cand must be 1, 2, 4, 8 or 16");
        n.lanes_per_cand = g;
    }
    if (t->visited_bits) {
        if (t->visited_bits < 8 || t->visited_bits > 13)
            return fail(LQG_ERR_ARG, "visited_bits must be in [8, 13]");
        n.visited_bits = t->visited_bits;
    }
    if (t->warps_per_block) {
        if (t->warps_per_block > 16) return fail(LQG_ERR_ARG, "warps_per_block must be <= 16");
        n.warps_per_block = t->warps_per_block;
    }
    if (t->blocks_per_sm) {
        if (t->blocks_per_sm > 32) return fail(LQG_ERR_ARG, "blocks_per_sm must be <= 32");
        n.blocks_per_sm = t->blocks_per_sm;
    }
    if (t->mode) {
        if (t->mode > 6) return fail(LQG_ERR_ARG, "mode must be in [1, 6]");
        n.mode = t->mode;
    }
    if (t->heap_warps) {
        if (t->heap_warps > 8) return fail(LQG_ERR_ARG, "heap_warps must be <= 8");
        n.heap_warps = t->heap_warps;
    }
    if (t->heap_scap) {
        if (t->heap_scap < 256 || t->heap_scap > 16384)
            return fail(LQG_ERR_ARG, "heap_scap must be in [256, 16384]");
        n.heap_scap = t->heap_scap;
    }
    n.replay_all = t->replay_all ? 1u : 0u;
    if (t->small_batch) n.small_batch = t->small_batch;
    if (t->replay_warps) {
        if (t->replay_warps > 15) return fail(LQG_ERR_ARG, "replay_warps must be in [1, 15]");
        n.replay_warps = t->replay_warps;
    }
    if (n.mode == 3 && lqg::replay_smem_bytes(ix->dim, n.visited_bits, n.heap_scap, 1) > 227 * 1024)
        return fail(LQG_ERR_ARG, "replay kernel tuning needs more than 227 KB of shared memory");
    if (n.mode == 4 && lqg::split_smem_bytes(ix->dim, n.visited_bits, n.heap_scap, 1) > 227 * 1024)
        return fail(LQG_ERR_ARG, "split kernel tuning needs more than 227 KB of shared memory");
    if (n.mode >= 5 && lqg::batch_smem_bytes(ix->dim, n.visited_bits, n.heap_scap,
                                             32u * (uint32_t)lqg::replay_pool_regs(kMaxEf), 1) >
                           227 * 1024)
        return fail(LQG_ERR_ARG, "batch kernel tuning needs more than 227 KB of shared memory");
    if (n.mode <= 2 &&
        lqg::heap_smem_bytes(ix->dim, n.visited_bits, kMaxEf + 2, n.heap_scap, (int)n.heap_warps) >
        227 * 1024)
        return fail(LQG_ERR_ARG, "heap kernel tuning needs more than 227 KB of shared memory");
    if (n.mode == 1 &&
        lqg::fast_smem_bytes(ix->dim, n.visited_bits, (int)n.warps_per_block) > 227 * 1024)
        return fail(LQG_ERR_ARG, "tuning needs more than 227 KB of shared memory per block");
    ix->tune = n;
    return LQG_OK;
}

lqg_status lqg_get_tuning(const lqg_index* ix, lqg_tuning* t) {
    if (!ix || !t) return fail(LQG_ERR_ARG, "null argument");
    *t = ix->tune;
    return LQG_OK;
}

lqg_status lqg_info(const lqg_index* ix, uint64_t* num_elements, uint32_t* dimension,
                    uint32_t* degree_bound, uint32_t* entry, uint32_t* ef) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (num_elements) *num_elements = ix->n;
    if (dimension) *dimension = ix->dim;
    if (degree_bound) *degree_bound = ix->deg;
    if (entry) *entry = ix->entry;
    if (ef) *ef = ix->ef;
    return LQG_OK;
}

lqg_status lqg_device_arrays(const lqg_index* ix, const uint32_t** nbrs, const uint8_t** codes,
                             const float** params, uint32_t* code_stride) {
    if (!ix) return fail(LQG_ERR_ARG, "null index");
    if (!ix->has_data) return fail(LQG_ERR_STATE, "index has no data");
    if (nbrs) *nbrs = ix->d_nbrs;
    if (codes) *codes = ix->d_codes;
    if (params) *params = ix->d_params;
    if (code_stride) *code_stride = ix->cstride;
    return LQG_OK;
}


// Index.build_index: python/bindings.cpp:69-90 -> QGBuilder
// (symqglib/qg/qg_builder.hpp:48-91), on the GPU:
//   SQ8 encode, entry = exact nearest point to the FP64 centroid, random
//   initial graph; then num_iter rounds of
//     search   every point through the current graph (fast search kernel,
//              pool of ef_build) — the candidate step of search_new_neighbors
//     prune    pool + current neighbours with exact FP32 distances (RNG rule)
//     reverse  add_reverse_edges: each kept edge offered to its target, the
//              target's list re-pruned, then filled to exactly degree_bound
//              with its pruned candidates and, if still short, random ids.
lqg_status lqg_build(lqg_index* ix, const float* data, uint32_t ef_build, uint32_t num_iter,
                     uint64_t seed, uint32_t random_edges) {
    return lqg_build_ex(ix, data, ef_build, num_iter, seed, random_edges, 1.0f, 0, 0, 1, nullptr);
}

lqg_status lqg_build_ex(lqg_index* ix, const float* data, uint32_t ef_build, uint32_t num_iter,
                        uint64_t seed, uint32_t random_edges, float alpha, uint32_t path_take,
                        uint32_t far_budget, uint32_t pair_kernel, lqg_build_report* report) {
    if (!ix || !data) return fail(LQG_ERR_ARG, "null argument");
    if (pair_kernel > 1) return fail(LQG_ERR_ARG, "pair_kernel must be 0 or 1");
    if (report) *report = lqg_build_report{};
    if (!(alpha >= 1.0f && alpha <= 4.0f)) return fail(LQG_ERR_ARG, "alpha must be in [1, 4]");
    if (path_take > 128) return fail(LQG_ERR_ARG, "path_take must be <= 128");
    if (far_budget + random_edges >= ix->deg)
        return fail(LQG_ERR_ARG, "far_budget + random_edges must be below degree_bound");
    const float alpha2 = alpha * alpha;
    if (num_iter <= 1) return fail(LQG_ERR_ARG, "The number of iter for building qg should >= 3");
    if (ef_build == 0 || ef_build > kMaxEf) return fail(LQG_ERR_ARG, "EF must be in [1, 512]");
    if (ix->n <= ix->deg) return fail(LQG_ERR_ARG, "num_elements must exceed degree_bound");
    if (random_edges >= ix->deg) return fail(LQG_ERR_ARG, "random_edges must be below degree_bound");
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    const uint64_t n = ix->n;
    const uint32_t dim = ix->dim, deg = ix->deg;
    try {
        ix->vectors.assign(data, data + n * dim);
        ix->nbrs.resize(n * deg);
        ix->codes.resize(n * dim);
        ix->params.resize(dim * 2);
    } catch (...) {
        return fail(LQG_ERR_NOMEM, "host allocation failed");
    }
    ix->has_data = false;
    dfree(ix->d_nbrs);
    dfree(ix->d_codes);
    dfree(ix->d_params);

    const uint32_t rest_stride = 64, rev_cap = deg;
    const uint64_t chunk = std::min<uint64_t>(n, 1u << 20);
    float* d_x = nullptr;
    uint8_t* d_c = nullptr;
    void* d_work = nullptr;
    float* d_cent = nullptr;
    unsigned long long* d_best = nullptr;
    uint32_t *d_kept = nullptr, *d_kept_cnt = nullptr, *d_rest = nullptr, *d_rest_cnt = nullptr;
    uint32_t *d_new = nullptr, *d_new_cnt = nullptr;
    lqg::ReverseWork rw{};
    uint32_t *d_pool = nullptr, *d_k1 = nullptr, *d_path = nullptr, *d_perr = nullptr;
    unsigned long long* d_rechk = nullptr;
    float* d_pool_d = nullptr;
    cudaEvent_t evb[4] = {nullptr, nullptr, nullptr, nullptr};
    double prune_ms = 0.0;
    // the build searches run the fast kernel with ties resolved by insertion order
    const lqg_tuning saved_tune = ix->tune;
    ix->tune.mode = 1;
    auto cleanup = [&]() {
        dfree(d_x); dfree(d_c); if (d_work) cudaFree(d_work); d_work = nullptr;
        dfree(d_cent); dfree(d_best); dfree(d_kept); dfree(d_kept_cnt); dfree(d_rest);
        dfree(d_rest_cnt); dfree(d_new); dfree(d_new_cnt);
        dfree(rw.keys_in); dfree(rw.vals_in); dfree(rw.keys_out); dfree(rw.vals_out);
        dfree(rw.start); dfree(rw.end); if (rw.temp) cudaFree(rw.temp); rw.temp = nullptr;
        dfree(d_pool); dfree(d_k1); dfree(d_pool_d); dfree(d_path); dfree(d_perr); dfree(d_rechk);
        for (auto& e : evb) if (e) { cudaEventDestroy(e); e = nullptr; }
        ix->tune = saved_tune;
    };
    auto alloc = [&](auto*& p, size_t bytes) {
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return false;
        }
        return true;
    };
    const size_t work_bytes = std::max(lqg::sq8_work_floats(dim) * sizeof(float),
                                       lqg::entry_work_doubles(dim) * sizeof(double));
    bool ok = alloc(d_x, n * dim * 4) && alloc(ix->d_codes, n * ix->cstride) &&
              alloc(ix->d_params, dim * 8) && alloc(ix->d_nbrs, n * deg * 4) &&
              alloc(d_work, work_bytes) && alloc(d_cent, dim * 4) && alloc(d_best, 8) &&
              alloc(d_kept, n * deg * 4) && alloc(d_kept_cnt, n * 4) &&
              alloc(d_rest, n * rest_stride * 4) && alloc(d_rest_cnt, n * 4) &&
              alloc(rw.keys_in, n * deg * 4) && alloc(rw.vals_in, n * deg * 4) &&
              alloc(rw.keys_out, n * deg * 4) && alloc(rw.vals_out, n * deg * 4) &&
              alloc(rw.start, n * 4) && alloc(rw.end, n * 4) &&
              alloc(rw.temp, (rw.temp_bytes = lqg::reverse_temp_bytes(n, deg)) + 256) &&
              alloc(d_new, n * deg * 4) && alloc(d_new_cnt, n * 4) &&
              alloc(d_pool, chunk * ef_build * 4) && alloc(d_pool_d, chunk * ef_build * 4) &&
              alloc(d_k1, chunk * 4) && (ix->cstride == dim || alloc(d_c, n * dim)) &&
              (path_take == 0 || alloc(d_path, chunk * path_take * 4)) && alloc(d_perr, 4) &&
              alloc(d_rechk, 8);
    if (!ok) {
        cleanup();
        return fail(LQG_ERR_NOMEM, "device allocation for the build failed");
    }
    cudaStream_t st = nullptr;
    for (auto& e : evb)
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            cleanup();
            return fail(LQG_ERR_CUDA, "event creation failed");
        }
    auto check_cuda = [&](cudaError_t e, const char* what) -> lqg_status {
        if (e == cudaSuccess) return LQG_OK;
        cleanup();
        return cuda_fail(e, what);
    };
    lqg_status s;
#define LQG_BCUDA(call, what) \
    if ((s = check_cuda((call), what)) != LQG_OK) return s
    LQG_BCUDA(cudaMemcpy(d_x, data, n * dim * 4, cudaMemcpyHostToDevice), "copy data");
    LQG_BCUDA(cudaMemset(d_perr, 0, 4), "build flags");
    LQG_BCUDA(cudaMemset(d_rechk, 0, 8), "build flags");
    LQG_BCUDA(cudaEventRecord(evb[0], st), "event");
    // prune launches are timed between evb[2] and evb[3]
    auto timed_prune = [&](const lqg::PruneArgs& pa, uint64_t nodes) -> cudaError_t {
        cudaError_t e = cudaEventRecord(evb[2], st);
        if (e == cudaSuccess) e = lqg::launch_prune(pa, nodes, st);
        if (e == cudaSuccess) e = cudaEventRecord(evb[3], st);
        if (e == cudaSuccess) e = cudaEventSynchronize(evb[3]);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, evb[2], evb[3]);
        prune_ms += ms;
        return e;
    };
    uint8_t* codes_out = ix->cstride == dim ? ix->d_codes : d_c;
    LQG_BCUDA(lqg::launch_sq8_encode(d_x, n, dim, ix->d_params, codes_out, (float*)d_work, st),
              "sq8 encode");
    if (ix->cstride != dim) {
        LQG_BCUDA(cudaMemset(ix->d_codes, 0, n * ix->cstride), "pad codes");
        LQG_BCUDA(cudaMemcpy2D(ix->d_codes, ix->cstride, d_c, dim, dim, n, cudaMemcpyDeviceToDevice),
                  "pad codes");
    }
    LQG_BCUDA(lqg::launch_entry(d_x, n, dim, (double*)d_work, d_cent, d_best, st), "entry point");
    unsigned long long best = 0;
    LQG_BCUDA(cudaMemcpy(&best, d_best, 8, cudaMemcpyDeviceToHost), "entry point");
    ix->entry = (uint32_t)(best & 0xFFFFFFFFull);
    LQG_BCUDA(lqg::launch_random_fill(ix->d_nbrs, nullptr, n, deg, seed, st), "random graph");
    ix->has_data = true;
    ix->fs.release();  // a new graph: any FastScan section is stale

    for (uint32_t it = 0; it < num_iter; ++it) {
        for (uint64_t c0 = 0; c0 < n; c0 += chunk) {
            const uint64_t m = std::min(chunk, n - c0);
            BatchSpec b{d_x + c0 * dim, (int64_t)m, nullptr, 1, nullptr, ef_build, d_k1, 1,
                        d_pool, d_pool_d, ef_build, nullptr, st, 1, d_path, path_take};
            if ((s = run_batch(ix, ix->ws, b, false)) != LQG_OK) {
                cleanup();
                return s;
            }
            if ((s = read_status(ix->ws, st)) != LQG_OK) {
                cleanup();
                return s;
            }
            lqg::PruneArgs a{};
            a.x = d_x;
            a.n = n;
            a.dim = dim;
            a.deg = deg;
            a.node0 = c0;
            a.pool = d_pool;
            a.pool_stride = ef_build;
            // candidates: pool, then search path, then the current list
            a.pool_take = std::min<uint32_t>(
                ef_build, std::max<int>(64, (int)lqg::kCandMax - (int)deg - (int)path_take));
            a.nb = ix->d_nbrs;
            a.out = d_kept;
            a.out_cnt = d_kept_cnt;
            a.rest = d_rest;
            a.rest_cnt = d_rest_cnt;
            a.rest_stride = rest_stride;
            a.alpha2 = alpha2;
            a.path = d_path;
            a.path_stride = path_take;
            a.path_take = path_take;
            a.far_take = std::min<uint32_t>(path_take, 32);
            a.far_budget = far_budget;
            a.pair_tc = (int)pair_kernel;
            a.err = d_perr;
            a.rechecks = d_rechk;
            LQG_BCUDA(timed_prune(a, m), "prune");
        }
        LQG_BCUDA(lqg::launch_reverse(d_kept, d_kept_cnt, n, deg, rw, st), "reverse edges");
        lqg::PruneArgs b{};
        b.x = d_x;
        b.n = n;
        b.dim = dim;
        b.deg = deg;
        b.node0 = 0;
        b.nb = d_kept;
        b.nb_cnt = d_kept_cnt;
        b.rev = rw.vals_out;
        b.rev_start = rw.start;
        b.rev_end = rw.end;
        b.rev_cap = rev_cap;
        b.out = d_new;
        b.out_cnt = d_new_cnt;
        b.out_cap = deg - random_edges;
        b.fill = 1;
        b.alpha2 = alpha2;
        b.far_budget = far_budget;
        b.rest_fill = d_rest;
        b.rest_fill_cnt = d_rest_cnt;
        b.rest_stride = rest_stride;
        b.pair_tc = (int)pair_kernel;
        b.err = d_perr;
        b.rechecks = d_rechk;
        LQG_BCUDA(timed_prune(b, n), "merge reverse edges");
        LQG_BCUDA(lqg::launch_random_fill(d_new, d_new_cnt, n, deg, seed + 1 + it, st), "fill");
        LQG_BCUDA(cudaMemcpy(ix->d_nbrs, d_new, n * deg * 4, cudaMemcpyDeviceToDevice), "graph");
    }
    LQG_BCUDA(cudaMemcpy(ix->nbrs.data(), ix->d_nbrs, n * deg * 4, cudaMemcpyDeviceToHost), "graph");
    LQG_BCUDA(cudaMemcpy2D(ix->codes.data(), dim, ix->d_codes, ix->cstride, dim, n,
                           cudaMemcpyDeviceToHost), "codes");
    LQG_BCUDA(cudaMemcpy(ix->params.data(), ix->d_params, dim * 8, cudaMemcpyDeviceToHost), "params");
    LQG_BCUDA(cudaEventRecord(evb[1], st), "event");
    LQG_BCUDA(cudaEventSynchronize(evb[1]), "event");
    uint32_t perr = 0;
    unsigned long long rechk = 0;
    LQG_BCUDA(cudaMemcpy(&perr, d_perr, 4, cudaMemcpyDeviceToHost), "build flags");
    LQG_BCUDA(cudaMemcpy(&rechk, d_rechk, 8, cudaMemcpyDeviceToHost), "build flags");
    if (report) {
        float bms = 0.f;
        cudaEventElapsedTime(&bms, evb[0], evb[1]);
        report->build_ms = bms;
        report->prune_ms = prune_ms;
        report->rechecks = rechk;
    }
#undef LQG_BCUDA
    if (perr) {
        cleanup();
        return fail(LQG_ERR_CUDA, "build: a tensor-core wait in the prune timed out");
    }
    cleanup();
    return validate_content(ix);
}

}  // extern "C"
