// Mid-near partners on the device: mid_near_pairs_dense of src/nndescent.cpp:731-768 (PaCMAP-style partners, the
// second closest of n_cand random rows, n_pairs times per row), with the reference's random streams and its
// squared-distance arithmetic, so the partners are the reference's own for the same thread count.
//
// The reference runs nt = min(n_threads, max(1, n / 2048)) threads; thread t walks rows [n t / nt, n (t + 1) / nt)
// with one generator Rng(seed + 48271 (t + 1)) and makes n_pairs x n_cand draws per row, in order. The draws never
// depend on the data, so the device splits the walk in two passes:
//  * mid_state_kernel: one thread per group of 64 rows of a stream jumps to the group's first draw and records
//    the generator state at each of its rows. xorshift64*'s state step is linear over GF(2), so k steps are one
//    64 x 64 bit matrix; the host builds the matrices of 2^b groups' worth of steps and a thread applies those of
//    the set bits of its group index.
//  * mid_pairs_kernel: one thread per (row, pair) steps its row's state to the pair's draws and keeps the two
//    smallest (squared distance, index), as the reference's partial_sort over std::pair does.
// The squared distance follows the reference's kernel for the host's instruction set (chosen at
// src/nndescent.cpp:101-106): AVX-512 (16 lanes of fused multiply-adds, lanes summed high half onto low half, the
// tail fused), AVX2 (8 lanes, ((0+1)+(2+3))+((4+5)+(6+7)), the tail fused) or the plain loop (4 interleaved sums,
// no fusion), each written with explicit rounding intrinsics so the compiler neither fuses nor reorders them.
#include "graph.cuh"
#include "sqdist.cuh"
#include <vector>
#include <thread>
#include <algorithm>
#include <cstdlib>

namespace mgb {

namespace {

constexpr int kGroup = 64;      // rows per thread of the state pass
constexpr int kJumpBits = 32;   // group indices below 2^32

__host__ __device__ __forceinline__ uint64_t xs_step(uint64_t s) {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    return s;
}

// a GF(2) linear map of 64-bit states as its 64 columns (column k = image of bit k)
struct BitMat {
    uint64_t col[64];
};
uint64_t apply_host(const BitMat& m, uint64_t s) {
    uint64_t r = 0;
    for (int k = 0; k < 64; ++k)
        if ((s >> k) & 1ull) r ^= m.col[k];
    return r;
}
BitMat compose(const BitMat& a, const BitMat& b) {   // a after b
    BitMat r;
    for (int k = 0; k < 64; ++k) r.col[k] = apply_host(a, b.col[k]);
    return r;
}
BitMat power(BitMat m, uint64_t e) {
    BitMat r;
    for (int k = 0; k < 64; ++k) r.col[k] = 1ull << k;
    while (e) {
        if (e & 1ull) r = compose(m, r);
        m = compose(m, m);
        e >>= 1;
    }
    return r;
}

// per stream: first row, row count, first group index (exclusive prefix), start state
struct StreamInfo {
    int64_t r0, rows, g0;
    uint64_t state;
};

__global__ void __launch_bounds__(256) mid_state_kernel(const uint64_t* __restrict__ jumps,
                                                        const StreamInfo* __restrict__ streams, int nt,
                                                        int64_t total_groups, int draws_per_row,
                                                        uint64_t* __restrict__ row_state) {
    __shared__ uint64_t J[kJumpBits * 64];
    for (int k = threadIdx.x; k < kJumpBits * 64; k += blockDim.x) J[k] = jumps[k];
    __syncthreads();
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= total_groups) return;
    int lo = 0, hi = nt - 1;   // the stream whose groups hold gid
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (streams[mid].g0 <= gid) lo = mid; else hi = mid - 1;
    }
    const StreamInfo st = streams[lo];
    const uint64_t g = (uint64_t)(gid - st.g0);
    uint64_t s = st.state;
    for (int b = 0; b < kJumpBits; ++b) {
        if (!((g >> b) & 1ull)) continue;
        uint64_t r = 0;
        const uint64_t* m = J + b * 64;
        for (int k = 0; k < 64; ++k)
            if ((s >> k) & 1ull) r ^= m[k];
        s = r;
    }
    const int64_t first = st.r0 + (int64_t)g * kGroup;
    const int64_t last = min(st.r0 + st.rows, first + kGroup);
    for (int64_t r = first; r < last; ++r) {
        row_state[r] = s;
        for (int t = 0; t < draws_per_row; ++t) s = xs_step(s);
    }
}

template <int ORDER>
__global__ void __launch_bounds__(256) mid_pairs_kernel(const float* __restrict__ X, int64_t n, int d, int n_pairs,
                                                        int n_cand, const uint64_t* __restrict__ row_state,
                                                        int32_t* __restrict__ out) {
    const int64_t total = n * n_pairs;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / n_pairs;
        const int p = (int)(t - i * n_pairs);
        Rng rng(0);
        rng.s = row_state[i];
        for (int k = 0; k < p * n_cand; ++k) rng.s = xs_step(rng.s);
        const float* xi = X + i * d;
        float d0 = 0.f, d1 = 0.f;
        int32_t j0 = -1, j1 = -1;
        for (int c = 0; c < n_cand; ++c) {
            int32_t j = (int32_t)rng.below((uint32_t)n);
            if (j == i) j = (int32_t)((j + 1) % n);
            const float dj = sqdist<ORDER>(xi, X + (int64_t)j * d, d);
            // (dist, index) in the order of std::pair's operator<: the two smallest so far
            if (j0 < 0 || dj < d0 || (dj == d0 && j < j0)) { d1 = d0; j1 = j0; d0 = dj; j0 = j; }
            else if (j1 < 0 || dj < d1 || (dj == d1 && j < j1)) { d1 = dj; j1 = j; }
        }
        out[t] = j1;
    }
}

}  // namespace

int host_distance_order() {
    // MAGNET_DISTANCE_ORDER (0, 1 or 2) reproduces another host's kernel
    if (const char* v = std::getenv("MAGNET_DISTANCE_ORDER"))
        if (*v >= '0' && *v <= '2' && v[1] == 0) return *v - '0';
#if defined(__x86_64__) || defined(__i386__)
    __builtin_cpu_init();
    if (__builtin_cpu_supports("avx512f")) return 0;
    if (__builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma")) return 1;
#endif
    return 2;
}

void mid_near_pairs_dev(const float* X, int64_t n, int d, int n_pairs, int n_cand, uint64_t seed, int n_threads,
                        int order, int32_t* out, GraphWork& w, cudaStream_t s) {
    const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(n_threads, std::max<int64_t>(1, n / 2048)));
    const int per_row = n_pairs * n_cand;
    // the state step as a matrix, and its powers for 2^b groups of rows
    BitMat T;
    for (int k = 0; k < 64; ++k) T.col[k] = xs_step(1ull << k);
    std::vector<uint64_t> tab(kJumpBits * 64);
    BitMat J = power(T, (uint64_t)kGroup * (uint64_t)per_row);
    for (int b = 0; b < kJumpBits; ++b) {
        std::copy(J.col, J.col + 64, tab.begin() + b * 64);
        J = compose(J, J);
    }
    std::vector<StreamInfo> streams(nt);
    int64_t groups = 0;
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t r0 = n * t / nt, r1 = n * (t + 1) / nt;
        streams[t] = {r0, r1 - r0, groups, Rng(seed + 48271ULL * (uint64_t)(t + 1)).s};
        groups += (r1 - r0 + kGroup - 1) / kGroup;
    }
    const size_t tab_bytes = tab.size() * sizeof(uint64_t);
    char* dev = static_cast<char*>(w.mid_tab.ensure(tab_bytes + streams.size() * sizeof(StreamInfo)));
    MGB_CUDA(cudaMemcpyAsync(dev, tab.data(), tab_bytes, cudaMemcpyHostToDevice, s));
    MGB_CUDA(cudaMemcpyAsync(dev + tab_bytes, streams.data(), streams.size() * sizeof(StreamInfo),
                             cudaMemcpyHostToDevice, s));
    uint64_t* row_state = static_cast<uint64_t*>(w.mid_state.ensure(sizeof(uint64_t) * (size_t)n));
    mid_state_kernel<<<(int)((groups + 255) / 256), 256, 0, s>>>(
        reinterpret_cast<const uint64_t*>(dev), reinterpret_cast<const StreamInfo*>(dev + tab_bytes), (int)nt, groups,
        per_row, row_state);
    MGB_LAUNCH_CHECK();
    const int64_t total = n * n_pairs;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 32LL * kNumSMs));
    if (order == 0) mid_pairs_kernel<0><<<blocks, 256, 0, s>>>(X, n, d, n_pairs, n_cand, row_state, out);
    else if (order == 1) mid_pairs_kernel<1><<<blocks, 256, 0, s>>>(X, n, d, n_pairs, n_cand, row_state, out);
    else mid_pairs_kernel<2><<<blocks, 256, 0, s>>>(X, n, d, n_pairs, n_cand, row_state, out);
    MGB_LAUNCH_CHECK();
    // the host tables are read by the copies above before they go out of scope
    MGB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace mgb
