// Dispatch of the replay search kernel over its pool-size instances.
#include "replay_kernel.cuh"

namespace lqg {

extern template cudaError_t replay_dispatch<2>(const SearchArgs&, const ReplayArgs&, int, int,
                                               int, cudaStream_t, int*);
extern template cudaError_t replay_dispatch<3>(const SearchArgs&, const ReplayArgs&, int, int,
                                               int, cudaStream_t, int*);
extern template cudaError_t replay_dispatch<5>(const SearchArgs&, const ReplayArgs&, int, int,
                                               int, cudaStream_t, int*);
extern template cudaError_t replay_dispatch<9>(const SearchArgs&, const ReplayArgs&, int, int,
                                               int, cudaStream_t, int*);
extern template cudaError_t replay_dispatch<17>(const SearchArgs&, const ReplayArgs&, int, int,
                                                int, cudaStream_t, int*);

// Smallest instance whose sorted pool holds ef entries plus 32 ties at the bound.
int replay_pool_regs(uint32_t ef_max) {
    const int es[] = {2, 3, 5, 9, 17};
    for (int e : es)
        if (32u * e - 32u >= ef_max) return e;
    return 0;
}

size_t replay_smem_bytes(uint32_t dim, uint32_t vbits, uint32_t scap, int swarps) {
    const size_t dpad = (dim + 15u) & ~15u;
    return 8 * dpad + (size_t)swarps * replay_warp_bytes(dim, vbits, scap);
}

cudaError_t launch_replay(const SearchArgs& a, const ReplayArgs& ra, int E, int G, int degw,
                          int blocks, cudaStream_t st, int* occ) {
    switch (E) {
        case 2: return replay_dispatch<2>(a, ra, G, degw, blocks, st, occ);
        case 3: return replay_dispatch<3>(a, ra, G, degw, blocks, st, occ);
        case 5: return replay_dispatch<5>(a, ra, G, degw, blocks, st, occ);
        case 9: return replay_dispatch<9>(a, ra, G, degw, blocks, st, occ);
        case 17: return replay_dispatch<17>(a, ra, G, degw, blocks, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lqg

namespace lqg {

// Result-heap replay pass (qg.hpp:329-343), one thread per query: the logged
// accepted nodes, in order, on a result heap laid out as GCC libstdc++ leaves
// it (push_heap: sift-up while comp(parent, value); pop_heap: hole from the
// root to a leaf along the larger child, the right one unless comp(right,
// left), then sift-up of the last element). Each push is checked against the
// reference's acceptance test on this heap (size < ef or top > distance), and
// the search warp's bound after it against rp.top(); then the output is the
// first k pops (results[k-1-j] = j-th pop) and, if asked, the whole pool in
// ascending order. Heaps live in shared memory, slot i of thread t at
// [i * blockDim + t]; a query that fails a check goes to the spill list.
__global__ void __launch_bounds__(32) rp_replay_kernel(SearchArgs a, ReplayArgs ra) {
    extern __shared__ uint2 hs[];
    const uint32_t T = blockDim.x;
    const int64_t qi = (int64_t)blockIdx.x * T + threadIdx.x;
    if (qi >= a.m) return;
    const uint32_t len = ra.rlen[qi];
    if (len == kNoId) return;  // the search failed: already on the spill list
    uint2* h = hs + threadIdx.x;
    auto key = [](uint2 x) { return __uint_as_float(x.y); };
    auto sift_up = [&](uint32_t hole, uint2 v) {
        while (hole > 0) {
            const uint32_t parent = (hole - 1) / 2;
            const uint2 p = h[parent * T];
            if (!(key(p) < key(v))) break;
            h[hole * T] = p;
            hole = parent;
        }
        h[hole * T] = v;
    };
    auto pop_top = [&](uint32_t n) {
        if (n <= 1) return;
        const uint32_t l = n - 1;
        const uint2 v = h[l * T];
        uint32_t hole = 0, second = 0;
        while (second < (l - 1) / 2) {
            second = 2 * (second + 1);
            const uint2 rr = h[second * T];
            const uint2 ll = h[(second - 1) * T];
            if (key(rr) < key(ll)) {
                --second;
                h[hole * T] = ll;
            } else {
                h[hole * T] = rr;
            }
            hole = second;
        }
        if ((l & 1u) == 0 && second == (l - 2) / 2) {
            second = 2 * (second + 1);
            h[hole * T] = h[(second - 1) * T];
            hole = second - 1;
        }
        sift_up(hole, v);
    };

    const uint32_t efq = a.efq ? a.efq[qi] : a.ef0;
    const uint32_t ef = min(max(efq, 1u), ra.efcap);
    const uint32_t k = min(a.kq ? a.kq[qi] : a.k0, a.kstride);
    const uint4* lg = ra.rlog + (size_t)qi * ra.rlog_cap;
    uint32_t n = 0;
    bool ok = len > 0 && len <= ra.rlog_cap;
    uint4 nx = ok ? lg[0] : make_uint4(0, 0, 0, 0);
    for (uint32_t i = 0; ok && i < len; ++i) {
        const uint4 e = nx;
        if (i + 1 < len) nx = lg[i + 1];
        const float y = __uint_as_float(e.y);
        if (!(n < ef || key(h[0]) > y)) {
            ok = false;
            break;
        }
        sift_up(n, make_uint2(e.x, e.y));
        ++n;
        if (n > ef) {
            pop_top(n);
            --n;
        }
        if (key(h[0]) != __uint_as_float(e.z)) ok = false;
    }
    if (!ok) {
        const uint32_t i = atomicAdd(ra.nspill, 1u);
        ra.spill[i] = (int32_t)qi;
        return;
    }
    // qg.hpp:340-343
    const uint32_t P = n, kk = min(k, P);
    uint32_t* out = a.ids + (size_t)qi * a.kstride;
    for (uint32_t x = 0; x < k - kk; ++x) out[x] = kNoId;
    if (a.pool_ids)
        for (uint32_t x = P; x < a.pstride; ++x) {
            a.pool_ids[(size_t)qi * a.pstride + x] = kNoId;
            a.pool_d[(size_t)qi * a.pstride + x] = CUDART_INF_F;
        }
    const uint32_t ex = a.pool_ids ? P : kk;
    for (uint32_t j = 0; j < ex; ++j) {
        const uint2 t = h[0];
        if (j < kk) out[k - 1 - j] = t.x;
        if (a.pool_ids && P - 1 - j < a.pstride) {
            a.pool_ids[(size_t)qi * a.pstride + (P - 1 - j)] = t.x;
            a.pool_d[(size_t)qi * a.pstride + (P - 1 - j)] = key(t);
        }
        pop_top(n);
        --n;
    }
}

cudaError_t launch_rp_replay(const SearchArgs& a, const ReplayArgs& ra, cudaStream_t st) {
    if (a.m <= 0) return cudaSuccess;
    constexpr int T = 32;
    const size_t smem = (size_t)ra.rcap * T * sizeof(uint2);
    cudaError_t e = cudaFuncSetAttribute(rp_replay_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t blocks = (a.m + T - 1) / T;
    rp_replay_kernel<<<(unsigned)blocks, T, smem, st>>>(a, ra);
    return cudaGetLastError();
}

}  // namespace lqg
