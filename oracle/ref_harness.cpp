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
//   * ref_fs_*: the upstream FastScan/RaBitQ path this fork still carries but
//     no longer calls, run on real data: FHTRotator::rotate with a given
//     diagonal (utils/rotator.hpp:89-114), QGQuery::query_prepare
//     (qg/qg_query.hpp:30-45), rabitq_codes (quantization/rabitq.hpp:23-59),
//     QGScanner::scan_neighbors (qg/qg_scanner.hpp:99-155), and
//     QuantizedGraph::search_qg (qg/qg.hpp:252-287) on an index whose rows are
//     laid out as upstream's (raw vector, packed codes, factors, neighbours).

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
#include "quantization/rabitq.hpp"
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

// ---- upstream FastScan / RaBitQ pieces ---------------------------------

static void set_diag(symqg::FHTRotator& r, const float* diag, size_t P) {
    for (size_t i = 0; i < P; ++i) r.mat_[i] = diag[i];
}

// dst[m][P] = rotator.rotate(src[m][dim]) with the rotator's diagonal = diag[P].
void ref_fs_rotate(uint64_t dim, const float* diag, const float* src, uint64_t m, float* dst) {
    symqg::FHTRotator rot(dim);
    const size_t P = rot.paded_dim_;
    set_diag(rot, diag, P);
    std::vector<float, symqg::memory::AlignedAllocator<float>> buf(P);
    for (uint64_t i = 0; i < m; ++i) {
        rot.rotate(src + i * dim, buf.data());
        std::copy(buf.begin(), buf.end(), dst + i * P);
    }
}

// QGQuery::query_prepare: lut[P*4], width, lower, sumq.
void ref_fs_query_prepare(uint64_t dim, uint64_t deg, const float* diag, const float* query,
                          uint8_t* lut, float* width, float* lower, int32_t* sumq) {
    symqg::FHTRotator rot(dim);
    const size_t P = rot.paded_dim_;
    set_diag(rot, diag, P);
    symqg::QGScanner scanner(P, deg);
    symqg::QGQuery q(query, P);
    q.query_prepare(rot, scanner);
    std::copy(q.lut().begin(), q.lut().end(), lut);
    *width = q.width();
    *lower = q.lower_val();
    *sumq = q.sumq();
}

// rabitq_codes of deg rotated neighbours (deg a multiple of 32) around a
// rotated centroid: packed[deg*P/8] in the FastScan block layout, factors[3][deg].
void ref_fs_rabitq(uint64_t P, uint64_t deg, const float* rot_nb, const float* rot_c,
                   uint8_t* packed, float* factors) {
    symqg::RowMatrix<float> x(deg, P), c(1, P);
    for (uint64_t i = 0; i < deg; ++i)
        for (uint64_t j = 0; j < P; ++j) x(i, j) = rot_nb[i * P + j];
    for (uint64_t j = 0; j < P; ++j) c(0, j) = rot_c[j];
    symqg::rabitq_codes(x, c, packed, factors, factors + deg, factors + 2 * deg);
}

// QGScanner::scan_neighbors: appro[deg] from a prepared query and one node's
// packed codes and factors.
void ref_fs_scan(uint64_t P, uint64_t deg, const uint8_t* lut, float sqr_y, float lower,
                 float width, int32_t sumq, const uint8_t* packed, const float* factors,
                 float* appro) {
    symqg::QGScanner scanner(P, deg);
    scanner.scan_neighbors(appro, lut, sqr_y, lower, width, sumq, packed, factors);
}

namespace {
struct FsIndex {
    std::unique_ptr<symqg::QuantizedGraph> master;
    std::vector<float> diag;
    size_t n = 0, dim = 0, deg = 0, P = 0;
};

// Upstream's row layout (qg.hpp:73-81): raw vector, packed codes, factors,
// neighbour ids; offsets in floats.
void fs_layout(symqg::QuantizedGraph& g, size_t dim, size_t deg, size_t P) {
    g.code_offset_ = dim;
    g.factor_offset_ = g.code_offset_ + deg * P / 32;
    g.neighbor_offset_ = g.factor_offset_ + 3 * deg;
    g.row_offset_ = g.neighbor_offset_ + deg;
}

struct FsView {
    symqg::QuantizedGraph g;
    float* own;
    FsView(const FsIndex& f) : g(1, f.deg, f.dim) {
        fs_layout(g, f.dim, f.deg, f.P);
        own = g.data_.pointer_;
        g.data_.pointer_ = const_cast<float*>(f.master->data_.pointer_);
        g.num_points_ = f.n;
        g.entry_point_ = f.master->entry_point_;
        set_diag(g.rotator_, f.diag.data(), f.P);
    }
    ~FsView() { g.data_.pointer_ = own; }
};
}  // namespace

// An upstream-layout index from arrays: vectors[n][dim], nbrs[n][deg],
// packed[n][deg*P/8] (FastScan blocks), factors[n][3][deg], diag[P].
void* ref_fs_open(uint64_t n, uint64_t dim, uint64_t deg, uint32_t entry, const float* vectors,
                  const uint32_t* nbrs, const uint8_t* packed, const float* factors,
                  const float* diag) {
    auto* f = new FsIndex();
    f->n = n;
    f->dim = dim;
    f->deg = deg;
    f->master = std::make_unique<symqg::QuantizedGraph>(n, deg, dim);
    auto& g = *f->master;
    f->P = g.padded_dim_;
    f->diag.assign(diag, diag + f->P);
    fs_layout(g, dim, deg, f->P);
    g.data_ = decltype(g.data_)(std::vector<size_t>{n, g.row_offset_});
    const size_t pb = deg * f->P / 8;
    for (uint64_t i = 0; i < n; ++i) {
        float* row = g.get_vector(i);
        std::copy(vectors + i * dim, vectors + (i + 1) * dim, row);
        std::memcpy(row + g.code_offset_, packed + i * pb, pb);
        std::copy(factors + i * 3 * deg, factors + (i + 1) * 3 * deg, row + g.factor_offset_);
        std::memcpy(row + g.neighbor_offset_, nbrs + i * deg, deg * sizeof(uint32_t));
    }
    g.entry_point_ = entry;
    return f;
}

void ref_fs_close(void* h) { delete static_cast<FsIndex*>(h); }

// search() as upstream wires it: visited_.clear(); search_pool_.clear();
// search_qg(query, k, results) (qg.hpp:235-243 with line 241 restored).
void ref_fs_search(void* h, const float* queries, int64_t m, int k, int ef, uint32_t* out_ids,
                   int nthreads) {
    auto* f = static_cast<FsIndex*>(h);
    int t = nthreads > 0 ? nthreads : static_cast<int>(std::thread::hardware_concurrency());
#pragma omp parallel num_threads(t)
    {
        FsView v(*f);
        v.g.set_ef(static_cast<size_t>(ef));
#pragma omp for schedule(dynamic, 8)
        for (int64_t i = 0; i < m; ++i) {
            v.g.visited_.clear();
            v.g.search_pool_.clear();
            v.g.search_qg(queries + i * f->dim, static_cast<uint32_t>(k), out_ids + i * k);
        }
    }
}

}  // extern "C"
