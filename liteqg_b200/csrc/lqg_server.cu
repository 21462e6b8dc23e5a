// Serving loop: continuous batching of single-query requests over one
// resident index.
//
// Requests arrive one at a time (lqg_server_submit, from any host thread).
// A dispatcher thread takes pending requests as soon as one of S stream
// contexts is free and launches them as one batch on that context's stream;
// requests that arrive while batches are on the GPU are admitted into the next
// free context, so their work overlaps with the batches in flight. A context
// owns everything a batch mutates on the device (its Workspace: control
// words, tie list, heap-kernel areas, per-query result and pop logs; and
// staging for the requests), which is what admission is measured against.
//
// Admission is by each request's own device state: a request's candidate and
// visited state is sized by its ef (the per-query logs of the batch kernel
// hold max(1024, 16 ef) entries), so requests are grouped in ef classes
// (ef <= 64, 128, 256, 512). A batch takes the oldest pending request and,
// in arrival order, every pending request of the same or a smaller class, up
// to the number of requests of that class whose state fits the context's
// share of the device budget. An ef-50 request therefore reserves an ef-64
// footprint, not an ef-512 one, and short requests are not held behind long
// ones of a larger class. A completer thread waits for batches in launch
// order, hands each request its ids and records its latency (arrival ->
// result; in lqg_server_replay the arrival is the scheduled one, so a client
// that falls behind its schedule shows in the latency).
//
// Each request is searched by the same kernels and with its own k and ef, so
// its result is exactly what a batched or single search of that query alone
// returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "lqg_host.h"
#include "lqg_internal.h"

using namespace lqg_host;
using Clock = std::chrono::steady_clock;

namespace {

struct Request {
    uint64_t ticket = 0;
    uint32_t k = 0, ef = 0;
    std::vector<float> q;
    std::vector<uint32_t> ids;
    // t_arrive: when the request arrived (the submit call, or its scheduled
    // arrival in lqg_server_replay); latency is measured from it
    Clock::time_point t_arrive, t_done;
    lqg_status status = LQG_OK;
    bool done = false;
};

struct Ctx {
    Workspace ws;
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    float* h_q = nullptr;  // pinned staging
    uint32_t* h_k = nullptr;
    uint32_t* h_ef = nullptr;
    uint32_t* h_ids = nullptr;
    uint32_t* h_ctl = nullptr;
    float* d_q = nullptr;
    uint32_t* d_k = nullptr;
    uint32_t* d_ef = nullptr;
    uint32_t* d_ids = nullptr;
    std::vector<Request*> batch;
    bool busy = false;
    lqg_status launch_status = LQG_OK;
};

}  // namespace

// ef classes of the admission: a request of ef e belongs to the first class
// whose bound is >= e.
constexpr uint32_t kEfClass[4] = {64, 128, 256, 512};
constexpr int kNumClass = 4;

struct lqg_server {
    lqg_index* ix = nullptr;
    lqg_server_config cfg{};
    uint32_t class_ef[kNumClass] = {};   // ef bound of each class (<= max_ef)
    uint32_t class_cap[kNumClass] = {};  // requests per batch of each class
    int nclass = 0;
    std::vector<Ctx> ctx;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> pending;
    std::deque<Ctx*> inflight;
    std::unordered_map<uint64_t, Request*> reqs;
    std::thread dispatcher, completer;
    bool stopping = false;
    bool dispatcher_done = false;
    uint64_t next_ticket = 1;
    // statistics
    std::vector<double> lat_us;
    uint64_t batches = 0, batched_queries = 0, completed = 0;
    Clock::time_point t_start;
    lqg_status fatal = LQG_OK;
};

namespace {

void free_ctx(Ctx& c, int device) {
    cudaSetDevice(device);
    c.ws.release();
    dfree(c.d_q);
    dfree(c.d_k);
    dfree(c.d_ef);
    dfree(c.d_ids);
    if (c.h_q) cudaFreeHost(c.h_q);
    if (c.h_k) cudaFreeHost(c.h_k);
    if (c.h_ef) cudaFreeHost(c.h_ef);
    if (c.h_ids) cudaFreeHost(c.h_ids);
    if (c.h_ctl) cudaFreeHost(c.h_ctl);
    if (c.ev) cudaEventDestroy(c.ev);
    if (c.st) cudaStreamDestroy(c.st);
    c = Ctx{};
}

int request_class(const lqg_server* s, uint32_t ef) {
    for (int i = 0; i < s->nclass; ++i)
        if (ef <= s->class_ef[i]) return i;
    return s->nclass - 1;
}

// Device bytes one request of ef bound `efc` holds while its batch runs:
// staging (query, k, ef, ids) and the batch kernel's per-query result log,
// pop log and log length.
size_t request_bytes(const lqg_index* ix, uint32_t max_k, uint32_t efc) {
    const size_t logs = (size_t)std::max(1024u, 16u * efc);
    return (size_t)ix->dim * 4 + (size_t)max_k * 4 + 8 + logs * (16 + 8) + 4;
}

void dispatch_loop(lqg_server* s) {
    cudaSetDevice(s->ix->device);
    const uint32_t dim = s->ix->dim;
    for (;;) {
        Ctx* c = nullptr;
        bool alone = false;  // no other batch in flight when this one launches
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                if (s->stopping && s->pending.empty()) return true;
                if (s->pending.empty()) return false;
                for (auto& x : s->ctx)
                    if (!x.busy) return true;
                return false;
            });
            if (s->stopping && s->pending.empty()) {
                s->dispatcher_done = true;
                s->cv_done.notify_all();
                return;
            }
            for (auto& x : s->ctx)
                if (!x.busy) {
                    c = &x;
                    break;
                }
            c->batch.clear();
            // the oldest request's class, then every pending request of that
            // class or a smaller one, in arrival order, up to the class's count
            const int c0 = request_class(s, s->pending.front()->ef);
            const uint32_t cap = s->class_cap[c0];
            std::deque<Request*> rest;
            while (!s->pending.empty()) {
                Request* r = s->pending.front();
                s->pending.pop_front();
                if (c->batch.size() < cap && request_class(s, r->ef) <= c0)
                    c->batch.push_back(r);
                else
                    rest.push_back(r);
                if (c->batch.size() == cap) break;
            }
            while (!rest.empty()) {  // put the skipped ones back, order kept
                s->pending.push_front(rest.back());
                rest.pop_back();
            }
            c->busy = true;
            alone = true;
            for (auto& x : s->ctx)
                if (&x != c && x.busy) alone = false;
        }
        const uint32_t m = (uint32_t)c->batch.size();
        uint32_t efmax = 1;
        for (uint32_t i = 0; i < m; ++i) {
            Request* r = c->batch[i];
            std::memcpy(c->h_q + (size_t)i * dim, r->q.data(), dim * sizeof(float));
            c->h_k[i] = r->k;
            c->h_ef[i] = r->ef;
            efmax = std::max(efmax, r->ef);
        }
        lqg_status st = LQG_OK;
        auto cu = [&](cudaError_t e, const char* what) {
            if (e != cudaSuccess && st == LQG_OK) st = cuda_fail(e, what);
        };
        cu(cudaMemcpyAsync(c->d_q, c->h_q, (size_t)m * dim * 4, cudaMemcpyHostToDevice, c->st), "H2D");
        cu(cudaMemcpyAsync(c->d_k, c->h_k, m * 4, cudaMemcpyHostToDevice, c->st), "H2D");
        cu(cudaMemcpyAsync(c->d_ef, c->h_ef, m * 4, cudaMemcpyHostToDevice, c->st), "H2D");
        if (st == LQG_OK) {
            BatchSpec b{c->d_q, (int64_t)m, c->d_k, 0, c->d_ef, efmax, c->d_ids,
                        s->cfg.max_k, nullptr, nullptr, 0, nullptr, c->st};
            // a batch that has the device to itself may run one query per
            // block (lower latency); under load the one-warp form keeps the
            // throughput
            b.small_ok = alone;
            st = run_batch(s->ix, c->ws, b, false);
        }
        if (st == LQG_OK) {
            cu(cudaMemcpyAsync(c->h_ids, c->d_ids, (size_t)m * s->cfg.max_k * 4,
                               cudaMemcpyDeviceToHost, c->st),
               "D2H");
            cu(cudaMemcpyAsync(c->h_ctl, c->ws.d_ctl, kCtlWords * 4, cudaMemcpyDeviceToHost, c->st),
               "D2H");
        }
        cu(cudaEventRecord(c->ev, c->st), "event");
        c->launch_status = st;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->inflight.push_back(c);
            ++s->batches;
            s->batched_queries += m;
        }
        s->cv_done.notify_all();
    }
}

void complete_loop(lqg_server* s) {
    cudaSetDevice(s->ix->device);
    for (;;) {
        Ctx* c = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_done.wait(lk, [&] {
                return !s->inflight.empty() || s->dispatcher_done;
            });
            if (s->inflight.empty()) return;
            c = s->inflight.front();
            s->inflight.pop_front();
        }
        lqg_status st = c->launch_status;
        if (cudaEventSynchronize(c->ev) != cudaSuccess && st == LQG_OK)
            st = fail(LQG_ERR_CUDA, "batch failed on the device");
        if (st == LQG_OK && c->h_ctl[kCtlErr]) st = LQG_ERR_CAPACITY;
        const auto now = Clock::now();
        // the batch's requests belong to this context until marked done: their
        // ids are copied outside the lock the submitters and waiters share
        for (size_t i = 0; i < c->batch.size(); ++i) {
            Request* r = c->batch[i];
            r->ids.assign(c->h_ids + i * s->cfg.max_k, c->h_ids + i * s->cfg.max_k + r->k);
            r->status = st;
            r->t_done = now;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t i = 0; i < c->batch.size(); ++i) {
                Request* r = c->batch[i];
                r->done = true;
                s->lat_us.push_back(
                    std::chrono::duration<double, std::micro>(now - r->t_arrive).count());
                ++s->completed;
            }
            c->batch.clear();
            c->busy = false;
        }
        s->cv_work.notify_all();
        s->cv_done.notify_all();
    }
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    const size_t i = std::min(v.size() - 1, (size_t)(p / 100.0 * (double)(v.size() - 1) + 0.5));
    std::nth_element(v.begin(), v.begin() + i, v.end());
    return v[i];
}

// One full-size batch of every class (its count of zero queries at max_k and
// the class's ef bound, in the index's current kernel mode) on context c
// before serving starts: the work areas a batch grows to fit (result and pop
// logs, work order, search-heap areas) reach their largest size here. Growing
// them while serving would free and allocate device memory, which waits for
// every stream of the device.
lqg_status warm_context(lqg_server* s, Ctx& c) {
    const uint32_t dim = s->ix->dim;
    for (int ci = 0; ci < s->nclass; ++ci) {
        const uint32_t mb = s->class_cap[ci];
        std::memset(c.h_q, 0, (size_t)mb * dim * sizeof(float));
        for (uint32_t i = 0; i < mb; ++i) {
            c.h_k[i] = s->cfg.max_k;
            c.h_ef[i] = s->class_ef[ci];
        }
        LQG_CUDA(cudaMemcpyAsync(c.d_q, c.h_q, (size_t)mb * dim * 4, cudaMemcpyHostToDevice, c.st));
        LQG_CUDA(cudaMemcpyAsync(c.d_k, c.h_k, (size_t)mb * 4, cudaMemcpyHostToDevice, c.st));
        LQG_CUDA(cudaMemcpyAsync(c.d_ef, c.h_ef, (size_t)mb * 4, cudaMemcpyHostToDevice, c.st));
        BatchSpec b{c.d_q, (int64_t)mb, c.d_k, 0, c.d_ef, s->class_ef[ci], c.d_ids,
                    s->cfg.max_k, nullptr, nullptr, 0, nullptr, c.st};
        b.small_ok = false;  // the one-warp form's work areas are the larger
        const lqg_status st = run_batch(s->ix, c.ws, b, false);
        if (st != LQG_OK) return st;
        LQG_CUDA(cudaStreamSynchronize(c.st));
    }
    return LQG_OK;
}

}  // namespace

extern "C" {

lqg_status lqg_server_start(lqg_index* ix, const lqg_server_config* cfg, lqg_server** out) {
    if (!ix || !out) return fail(LQG_ERR_ARG, "null argument");
    *out = nullptr;
    if (!ix->has_data) return fail(LQG_ERR_STATE, "index has no data");
    lqg_server_config c = cfg ? *cfg : lqg_server_config{};
    if (c.streams == 0) c.streams = 4;
    if (c.max_k == 0) c.max_k = 100;
    if (c.max_ef == 0) c.max_ef = kMaxEf;
    if (c.max_ef > kMaxEf) return fail(LQG_ERR_ARG, "max_ef must be <= 512");
    if (c.streams > 64) return fail(LQG_ERR_ARG, "streams must be <= 64");
    DeviceScope ds(ix->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    auto* s = new (std::nothrow) lqg_server();
    if (!s) return fail(LQG_ERR_NOMEM, "host allocation failed");
    s->ix = ix;
    // ef classes up to max_ef; each class's count from the context's share of
    // the budget and its requests' footprint (max_batch, if set, caps it)
    const uint64_t budget = c.state_budget ? c.state_budget : (4ull << 30);
    uint32_t most = 1;
    for (uint32_t b : kEfClass) {
        const uint32_t efc = std::min(b, c.max_ef);
        if (s->nclass > 0 && s->class_ef[s->nclass - 1] >= efc) break;
        uint64_t cnt = std::max<uint64_t>(1, budget / c.streams / request_bytes(ix, c.max_k, efc));
        cnt = std::min<uint64_t>(cnt, 16384);
        if (c.max_batch) cnt = std::min<uint64_t>(cnt, c.max_batch);
        s->class_ef[s->nclass] = efc;
        s->class_cap[s->nclass] = (uint32_t)cnt;
        most = std::max(most, (uint32_t)cnt);
        ++s->nclass;
    }
    c.max_batch = most;  // staging size: the largest class count
    s->cfg = c;
    s->ctx.resize(c.streams);
    for (auto& x : s->ctx) {
        const size_t mb = c.max_batch;
        bool ok = cudaStreamCreateWithFlags(&x.st, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&x.ev, cudaEventDisableTiming) == cudaSuccess &&
                  cudaMallocHost(&x.h_q, mb * ix->dim * 4) == cudaSuccess &&
                  cudaMallocHost(&x.h_k, mb * 4) == cudaSuccess &&
                  cudaMallocHost(&x.h_ef, mb * 4) == cudaSuccess &&
                  cudaMallocHost(&x.h_ids, mb * c.max_k * 4) == cudaSuccess &&
                  cudaMallocHost(&x.h_ctl, kCtlWords * 4) == cudaSuccess &&
                  cudaMalloc(&x.d_q, mb * ix->dim * 4) == cudaSuccess &&
                  cudaMalloc(&x.d_k, mb * 4) == cudaSuccess &&
                  cudaMalloc(&x.d_ef, mb * 4) == cudaSuccess &&
                  cudaMalloc(&x.d_ids, mb * c.max_k * 4) == cudaSuccess &&
                  ensure_ctl(x.ws, (int64_t)mb) == LQG_OK &&
                  ensure_exact(x.ws, std::max(1, ix->num_sms / 4), 4) == LQG_OK;
        if (!ok) {
            cudaGetLastError();
            for (auto& y : s->ctx) free_ctx(y, ix->device);
            delete s;
            return fail(LQG_ERR_NOMEM, "serving-loop context allocation failed");
        }
    }
    for (auto& x : s->ctx) {
        const lqg_status st = warm_context(s, x);
        if (st != LQG_OK) {
            for (auto& y : s->ctx) free_ctx(y, ix->device);
            delete s;
            return st;
        }
    }
    s->t_start = Clock::now();
    s->dispatcher = std::thread(dispatch_loop, s);
    s->completer = std::thread(complete_loop, s);
    *out = s;
    return LQG_OK;
}

lqg_status lqg_server_submit(lqg_server* s, const float* query, uint32_t k, uint32_t ef,
                             uint64_t* ticket) {
    if (!s || !query || !ticket) return fail(LQG_ERR_ARG, "null argument");
    if (k == 0 || k > s->cfg.max_k) return fail(LQG_ERR_ARG, "k must be in [1, max_k]");
    if (ef == 0) ef = s->ix->ef;
    if (ef == 0 || ef > s->cfg.max_ef) return fail(LQG_ERR_ARG, "ef must be in [1, max_ef] (or set_ef)");
    auto* r = new (std::nothrow) Request();
    if (!r) return fail(LQG_ERR_NOMEM, "host allocation failed");
    r->k = k;
    r->ef = ef;
    r->q.assign(query, query + s->ix->dim);
    r->t_arrive = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) {
            delete r;
            return fail(LQG_ERR_STATE, "server is stopping");
        }
        r->ticket = s->next_ticket++;
        s->reqs[r->ticket] = r;
        s->pending.push_back(r);
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return LQG_OK;
}

lqg_status lqg_server_wait(lqg_server* s, uint64_t ticket, uint32_t* ids, int64_t timeout_us,
                           double* latency_us) {
    if (!s) return fail(LQG_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(LQG_ERR_ARG, "unknown ticket");
    Request* r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_us < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready)) {
        return fail(LQG_ERR_STATE, "timed out");
    }
    if (ids) std::memcpy(ids, r->ids.data(), r->ids.size() * 4);
    if (latency_us) *latency_us = std::chrono::duration<double, std::micro>(r->t_done - r->t_arrive).count();
    lqg_status st = r->status;
    s->reqs.erase(it);
    delete r;
    if (st == LQG_ERR_CAPACITY) return fail(st, "a query of this request's batch overflowed a work area");
    if (st != LQG_OK) return fail(st, "batch failed");
    return LQG_OK;
}

lqg_status lqg_server_replay(lqg_server* s, const float* queries, int64_t m, const uint32_t* k,
                             const uint32_t* ef, const double* arrival_us, uint32_t* ids,
                             uint32_t kstride, double* latency_us) {
    if (!s || !queries || !k || !ef || !ids) return fail(LQG_ERR_ARG, "null argument");
    std::vector<std::atomic<uint64_t>> tickets((size_t)m);
    for (auto& t : tickets) t.store(0);
    std::atomic<int> err{LQG_OK};
    std::atomic<int64_t> submitted{0};
    // the client submits, under one lock, every request whose arrival time
    // has come (up to 1,024 at once), and stamps each with its scheduled
    // arrival, so a client that falls behind shows as latency, not as a lower
    // offered rate
    std::thread client([&] {
        const auto t0 = Clock::now();
        auto due_of = [&](int64_t i) {
            return t0 + std::chrono::duration_cast<Clock::duration>(
                            std::chrono::duration<double, std::micro>(arrival_us[i]));
        };
        std::vector<Request*> group;
        int64_t i = 0;
        while (i < m) {
            if (arrival_us) {
                const auto due = due_of(i);
                while (Clock::now() < due) {
                    const auto left = due - Clock::now();
                    if (left > std::chrono::microseconds(200)) std::this_thread::sleep_for(left / 2);
                }
            }
            const auto now = Clock::now();
            int64_t j = i + 1;
            if (arrival_us)
                while (j < m && j - i < 1024 && due_of(j) <= now) ++j;
            group.clear();
            for (int64_t x = i; x < j; ++x) {
                const uint32_t kx = k[x], efx = ef[x] ? ef[x] : s->ix->ef;
                if (kx == 0 || kx > s->cfg.max_k || efx == 0 || efx > s->cfg.max_ef) {
                    err.store(fail(LQG_ERR_ARG, "request k or ef out of range"));
                    tickets[(size_t)x].store(~0ull);
                    group.push_back(nullptr);
                    continue;
                }
                auto* r = new (std::nothrow) Request();
                if (!r) {
                    err.store(fail(LQG_ERR_NOMEM, "host allocation failed"));
                    tickets[(size_t)x].store(~0ull);
                    group.push_back(nullptr);
                    continue;
                }
                r->k = kx;
                r->ef = efx;
                r->q.assign(queries + (size_t)x * s->ix->dim, queries + (size_t)(x + 1) * s->ix->dim);
                r->t_arrive = arrival_us ? due_of(x) : now;
                group.push_back(r);
            }
            {
                std::lock_guard<std::mutex> lk(s->mu);
                for (int64_t x = i; x < j; ++x) {
                    Request* r = group[(size_t)(x - i)];
                    if (!r) continue;
                    if (s->stopping) {
                        delete r;
                        group[(size_t)(x - i)] = nullptr;
                        err.store(fail(LQG_ERR_STATE, "server is stopping"));
                        tickets[(size_t)x].store(~0ull);
                        continue;
                    }
                    r->ticket = s->next_ticket++;
                    s->reqs[r->ticket] = r;
                    s->pending.push_back(r);
                }
            }
            s->cv_work.notify_one();
            for (int64_t x = i; x < j; ++x)
                if (Request* r = group[(size_t)(x - i)]) tickets[(size_t)x].store(r->ticket);
            submitted.store(j);
            i = j;
        }
    });
    // collect in submission order (each wait blocks until that ticket exists and is done)
    for (int64_t i = 0; i < m; ++i) {
        uint64_t t;
        while ((t = tickets[(size_t)i].load()) == 0) std::this_thread::yield();
        if (t == ~0ull) continue;
        double lat = 0;
        lqg_status st = lqg_server_wait(s, t, ids + (size_t)i * kstride, -1, &lat);
        if (st != LQG_OK) err.store(st);
        if (latency_us) latency_us[i] = lat;
    }
    client.join();
    return (lqg_status)err.load();
}

lqg_status lqg_server_stats(lqg_server* s, lqg_server_metrics* out) {
    if (!s || !out) return fail(LQG_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = s->completed;
    out->batches = s->batches;
    out->mean_batch = s->batches ? (double)s->batched_queries / (double)s->batches : 0.0;
    out->p50_us = percentile(s->lat_us, 50);
    out->p99_us = percentile(s->lat_us, 99);
    const double el = std::chrono::duration<double>(Clock::now() - s->t_start).count();
    out->qps = el > 0 ? (double)s->completed / el : 0.0;
    out->max_batch = s->cfg.max_batch;
    out->streams = s->cfg.streams;
    return LQG_OK;
}

lqg_status lqg_server_reset_stats(lqg_server* s) {
    if (!s) return fail(LQG_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat_us.clear();
    s->batches = s->batched_queries = s->completed = 0;
    s->t_start = Clock::now();
    return LQG_OK;
}

lqg_status lqg_server_stop(lqg_server* s) {
    if (!s) return LQG_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    s->cv_done.notify_all();
    if (s->completer.joinable()) s->completer.join();
    for (auto& x : s->ctx) free_ctx(x, s->ix->device);
    for (auto& kv : s->reqs) delete kv.second;
    delete s;
    return LQG_OK;
}

}  // extern "C"
