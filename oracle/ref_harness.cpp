// Test infrastructure: a C-ABI harness around the UNMODIFIED reference search
// and build code (LiteQG / SymphonyQG fork, header-only C++ under symqglib/).
//
// This file contains no reference source. It is compiled against the reference
// headers where they lie (see oracle/Makefile) into oracle/_ref/, and is used
// only by tests/ (to pin the C oracle restatement and to generate golden
// vectors) and by bench.py's CPU-baseline / reference arm. Nothing in the
// product library links or loads it.
//
// What it exposes:
//   * ref_open / ref_close: QuantizedGraph::load_index (symqglib/qg/qg.hpp:217-224).
//   * ref_search: QuantizedGraph::set_ef + QuantizedGraph::search
//     (symqglib/qg/qg.hpp:226-243), over M queries, on T OpenMP threads. The
//     reference search is not re-entrant (it owns one visited set,
//     qg.hpp:70,302), so each thread gets its own QuantizedGraph "view" whose
//     vector/code arrays alias the loaded index (no copy). Each call is exactly
//     the reference's own single-query search.
//   * ref_build: QGBuilder + QuantizedGraph::save_index (qg_builder.hpp:48-91,
//     qg.hpp:206-215), i.e. what symphonyqg.Index.build_index + save do.
//   * ref_sq8_quantize / ref_sq8_l2: the reference SQ8 encoder and the
//     decode+L2 used per neighbour (sq8.hpp:11-32, l2.hpp:16-59).
//   * ref_isa: which l2_sqr branch this build took (16 = AVX-512, 8 = AVX2).

// Standard headers first, so that the access override below only reaches the
// reference's own classes.
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>

#include <algorithm>
#include <array>
#include <cassert>
#include <cfloat>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <queue>
#include <random>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "common.hpp"  // pulls in Eigen before the override

// The harness needs the index's private arrays to alias them across threads.
#define private public
#include "qg/qg.hpp"
#include "qg/qg_builder.hpp"
#undef private

namespace {

struct RefIndex {
    std::unique_ptr<symqg::QuantizedGraph> master;
    size_t n = 0, dim = 0, deg = 0;
};

// A per-thread view: its own visited set and heaps, the master's arrays.
struct View {
    symqg::QuantizedGraph g;
    float* own_data;
    uint8_t* own_qdata;
    View(const symqg::QuantizedGraph& m, size_t dim, size_t deg)
        : g(1, deg, dim) {
        own_data = g.data_.pointer_;
        own_qdata = g.qdata_.pointer_;
        g.data_.pointer_ = const_cast<float*>(m.data_.pointer_);
        g.qdata_.pointer_ = const_cast<uint8_t*>(m.qdata_.pointer_);
        g.num_points_ = m.num_points_;
        g.entry_point_ = m.entry_point_;
        g.sq8_params_ = m.sq8_params_;
    }
    ~View() {
        g.data_.pointer_ = own_data;
        g.qdata_.pointer_ = own_qdata;
    }
};

}  // namespace

extern "C" {

int ref_isa() {
#if defined(__AVX512F__)
    return 16;
#elif defined(__AVX2__)
    return 8;
#else
    return 1;
#endif
}

void* ref_open(const char* path, uint64_t n, uint64_t dim, uint64_t deg) {
    auto* r = new RefIndex();
    r->n = n;
    r->dim = dim;
    r->deg = deg;
    r->master = std::make_unique<symqg::QuantizedGraph>(n, deg, dim);
    r->master->load_index(path);
    return r;
}

void ref_close(void* h) { delete static_cast<RefIndex*>(h); }

uint32_t ref_entry_point(void* h) {
    return static_cast<RefIndex*>(h)->master->entry_point_;
}

// out_ids[M*k] is pre-filled by the caller; slots the reference leaves
// unwritten (pool smaller than k) keep the caller's fill value.
// nthreads <= 0 means all hardware threads.
void ref_search(
    void* h,
    const float* queries,
    int64_t m,
    int k,
    int ef,
    uint32_t* out_ids,
    int nthreads
) {
    auto* r = static_cast<RefIndex*>(h);
    int t = nthreads > 0 ? nthreads : static_cast<int>(std::thread::hardware_concurrency());
    if (t <= 1) {
        View v(*r->master, r->dim, r->deg);
        v.g.set_ef(static_cast<size_t>(ef));
        for (int64_t i = 0; i < m; ++i) {
            v.g.search(queries + i * r->dim, static_cast<uint32_t>(k), out_ids + i * k);
        }
        return;
    }
#pragma omp parallel num_threads(t)
    {
        View v(*r->master, r->dim, r->deg);
        v.g.set_ef(static_cast<size_t>(ef));
#pragma omp for schedule(dynamic, 16)
        for (int64_t i = 0; i < m; ++i) {
            v.g.search(queries + i * r->dim, static_cast<uint32_t>(k), out_ids + i * k);
        }
    }
}

// Builds with the reference builder and saves to path. Returns 0.
int ref_build(
    const float* data,
    uint64_t n,
    uint64_t dim,
    uint64_t deg,
    uint64_t ef_build,
    uint64_t num_iter,
    int nthreads,
    const char* path
) {
    symqg::QuantizedGraph qg(n, deg, dim);
    size_t t = nthreads > 0 ? static_cast<size_t>(nthreads) : UINT_MAX;
    symqg::QGBuilder builder(qg, static_cast<uint32_t>(ef_build), data, t);
    builder.build(num_iter);
    qg.save_index(path);
    return 0;
}

void ref_sq8_quantize(
    const float* data, uint64_t dim, uint64_t n, uint8_t* codes, float* params
) {
    symqg::sq8_quantize(
        data, dim, n, codes, reinterpret_cast<symqg::SQ8Params*>(params)
    );
}

// dist[i] = l2_sqr(query, sq8_dequantize(codes[i])) exactly as one
// search_qg_with_heap neighbour evaluation (qg.hpp:325-328).
void ref_sq8_l2(
    const float* query,
    const uint8_t* codes,
    uint64_t n,
    uint64_t dim,
    const float* params,
    float* dist
) {
    std::vector<float> dec(dim);
    const auto* p = reinterpret_cast<const symqg::SQ8Params*>(params);
    for (uint64_t i = 0; i < n; ++i) {
        symqg::sq8_dequantize(codes + i * dim, dim, dec.data(), p);
        dist[i] = symqg::space::l2_sqr(query, dec.data(), dim);
    }
}

}  // extern "C"
