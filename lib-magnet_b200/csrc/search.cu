// Query kNN on the device: knn_search of src/nndescent.cpp:585-690 (the beam search of new rows over the training
// rows' neighbour graph that MAGNET.transform runs, magnet/knn.py:131-152).
//
// Per query the reference keeps a max-heap of the best `ef` rows found (res), a min-heap of rows still to expand
// (cand) and a visited stamp per row; it starts from the n_entry landmarks closest to the query (or n_entry random
// rows without landmarks), then repeatedly expands the closest candidate's graph row until the closest candidate is
// farther than the ef-th result. Here one warp runs one query with the same steps:
//  * the distances of a graph row's neighbours (or of the landmarks) are computed by the warp's lanes at once, in
//    the reference's squared-distance order (sqdist.cuh), so every distance equals the reference's bit for bit;
//  * the visited marks are a bit per training row in a bitset owned by the warp (test-and-set with atomicOr, the
//    row's neighbours at once; the rows of a CSR row are distinct), cleared after the query from its visit list;
//  * the decisions (is the row better than the ef-th result, push it on both heaps) are then taken by one lane in
//    the row's order, as the reference's loop takes them, with both heaps in shared memory.
// The expansion order and the result set therefore follow the reference's exactly whenever no two distances tie
// (ties may be broken differently by the two heap implementations). The results are sorted by (distance, row).
#include "common.cuh"
#include "sqdist.cuh"
#include "graph.cuh"
#include <vector>
#include <algorithm>
#include <string>

namespace mgb {

namespace {

constexpr int kSearchWarps = 4;        // queries in flight per block
constexpr int kMaxEf = 256;            // result heap capacity (ef)
constexpr int kCandCap = 2048;         // candidate heap capacity; a query that needs more is reported
constexpr int kVisitCap = 16384;       // visit list per warp; past it the warp clears its whole bitset

struct Entry {
    float d;
    int32_t i;
};

struct WarpHeaps {
    Entry res[kMaxEf + 1];   // one over while the ef-th result is replaced
    Entry cand[kCandCap];
};

// max-heap on d (res) and min-heap on d (cand), one lane
__device__ __forceinline__ void res_push(Entry* h, int& n, Entry e) {
    int c = n++;
    while (c > 0) {
        const int p = (c - 1) >> 1;
        if (!(h[p].d < e.d)) break;
        h[c] = h[p];
        c = p;
    }
    h[c] = e;
}
__device__ __forceinline__ void res_pop(Entry* h, int& n) {
    const Entry e = h[--n];
    int c = 0;
    for (;;) {
        int l = 2 * c + 1;
        if (l >= n) break;
        if (l + 1 < n && h[l].d < h[l + 1].d) ++l;
        if (!(e.d < h[l].d)) break;
        h[c] = h[l];
        c = l;
    }
    if (n > 0) h[c] = e;
}
__device__ __forceinline__ void cand_push(Entry* h, int& n, Entry e) {
    int c = n++;
    while (c > 0) {
        const int p = (c - 1) >> 1;
        if (!(e.d < h[p].d)) break;
        h[c] = h[p];
        c = p;
    }
    h[c] = e;
}
__device__ __forceinline__ Entry cand_pop(Entry* h, int& n) {
    const Entry top = h[0];
    const Entry e = h[--n];
    int c = 0;
    for (;;) {
        int l = 2 * c + 1;
        if (l >= n) break;
        if (l + 1 < n && h[l + 1].d < h[l].d) ++l;
        if (!(h[l].d < e.d)) break;
        h[c] = h[l];
        c = l;
    }
    if (n > 0) h[c] = e;
    return top;
}

__device__ __forceinline__ bool pair_less(float da, int32_t ia, float db, int32_t ib) {
    return da < db || (da == db && ia < ib);
}

struct SearchArgs {
    const float* X; int64_t n; int d;
    const int32_t* gptr; const int32_t* gidx;
    const int32_t* land; int64_t n_land;
    const int32_t* entries;            // m x n_entry random entry rows (no landmarks), else null
    const float* Q; int64_t m;
    int k, ef, n_entry;
    int32_t* out_i; float* out_d;
    uint32_t* bits; int64_t bit_words;   // per warp slot: bit_words words
    int32_t* visits;                      // per warp slot: kVisitCap rows
    float* ldist;                         // per warp slot: n_land distances
    int* overflow;                        // queries whose candidate heap filled up
};

template <int ORDER>
__global__ void __launch_bounds__(32 * kSearchWarps) search_kernel(SearchArgs a) {
    extern __shared__ unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    WarpHeaps& H = reinterpret_cast<WarpHeaps*>(smem_raw)[wib];
    const int64_t slot = (int64_t)blockIdx.x * kSearchWarps + wib;
    const int64_t slots = (int64_t)gridDim.x * kSearchWarps;
    uint32_t* bits = a.bits + slot * a.bit_words;
    int32_t* visits = a.visits + slot * kVisitCap;
    float* ldist = a.ldist + slot * a.n_land;
    for (int64_t q = slot; q < a.m; q += slots) {
        const float* qv = a.Q + q * a.d;
        int nres = 0, ncand = 0, nvis = 0;
        bool overflow = false;
        // rows of one batch (up to 32, one per lane) in the reference's order: distance, visited test-and-set,
        // then the sequential decisions of consider() on lane 0
        auto consider_batch = [&](int32_t j, bool valid) {
            float dd = 0.f;
            bool fresh = false;
            if (valid) {
                const uint32_t bit = 1u << (j & 31);
                fresh = (atomicOr(&bits[j >> 5], bit) & bit) == 0u;
                if (fresh) dd = sqdist<ORDER>(qv, a.X + (int64_t)j * a.d, a.d);
            }
            const unsigned fm = __ballot_sync(0xffffffffu, fresh);
            if (fresh) {
                const int r = nvis + __popc(fm & ((1u << lane) - 1u));
                if (r < kVisitCap) visits[r] = j;
            }
            nvis += __popc(fm);
            unsigned mm = fm;
            while (mm) {
                const int src = __ffs(mm) - 1;
                mm &= mm - 1u;
                const float dj = __shfl_sync(0xffffffffu, dd, src);
                const int32_t jj = __shfl_sync(0xffffffffu, j, src);
                if (lane == 0) {
                    if (nres < a.ef || dj < H.res[0].d) {
                        res_push(H.res, nres, Entry{dj, jj});
                        if (nres > a.ef) res_pop(H.res, nres);
                        if (ncand < kCandCap) cand_push(H.cand, ncand, Entry{dj, jj});
                        else overflow = true;
                    }
                }
            }
            nres = __shfl_sync(0xffffffffu, nres, 0);
            ncand = __shfl_sync(0xffffffffu, ncand, 0);
        };
        // entry points
        if (a.n_land > 0) {
            for (int64_t l = lane; l < a.n_land; l += 32) ldist[l] = sqdist<ORDER>(qv, a.X + (int64_t)a.land[l] * a.d, a.d);
            __syncwarp();
            const int take = (int)((int64_t)a.n_entry < a.n_land ? (int64_t)a.n_entry : a.n_land);
            float last_d = -INFINITY;
            int32_t last_i = -1;
            for (int e = 0; e < take; ++e) {
                // the next (distance, row) pair after the last one taken: the partial_sort of the reference
                float bd = INFINITY;
                int32_t bi = INT32_MAX;
                for (int64_t l = lane; l < a.n_land; l += 32) {
                    const float dl = ldist[l];
                    const int32_t il = a.land[l];
                    if (pair_less(last_d, last_i, dl, il) && pair_less(dl, il, bd, bi)) { bd = dl; bi = il; }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const float od = __shfl_xor_sync(0xffffffffu, bd, o);
                    const int32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (pair_less(od, oi, bd, bi)) { bd = od; bi = oi; }
                }
                last_d = bd; last_i = bi;
                consider_batch(bi, lane == 0);
            }
        } else {
            for (int e = 0; e < a.n_entry; ++e) consider_batch(a.entries[q * a.n_entry + e], lane == 0);
        }
        // expansions
        for (;;) {
            __syncwarp();
            if (ncand == 0) break;
            Entry c{0.f, 0};
            if (lane == 0) c = cand_pop(H.cand, ncand);
            __syncwarp();
            ncand = __shfl_sync(0xffffffffu, ncand, 0);
            c.d = __shfl_sync(0xffffffffu, c.d, 0);
            c.i = __shfl_sync(0xffffffffu, c.i, 0);
            const float worst = __shfl_sync(0xffffffffu, lane == 0 ? H.res[0].d : 0.f, 0);
            if (nres >= a.ef && c.d > worst) break;
            const int32_t b = a.gptr[c.i], e = a.gptr[c.i + 1];
            for (int32_t j0 = b; j0 < e; j0 += 32) {
                const int32_t j = j0 + lane < e ? a.gidx[j0 + lane] : 0;
                consider_batch(j, j0 + lane < e);
            }
        }
        __syncwarp();
        // results sorted by (distance, row); the first k
        if (lane == 0) {
            for (int x = 1; x < nres; ++x) {
                const Entry v = H.res[x];
                int y = x - 1;
                while (y >= 0 && pair_less(v.d, v.i, H.res[y].d, H.res[y].i)) { H.res[y + 1] = H.res[y]; --y; }
                H.res[y + 1] = v;
            }
            if (overflow) atomicAdd(a.overflow, 1);
        }
        __syncwarp();
        for (int c = lane; c < a.k; c += 32) {
            a.out_i[q * a.k + c] = c < nres ? H.res[c].i : -1;
            a.out_d[q * a.k + c] = c < nres ? H.res[c].d : INFINITY;
        }
        // clear this query's visited bits for the next one
        if (nvis <= kVisitCap) {
            for (int v = lane; v < nvis; v += 32) bits[visits[v] >> 5] = 0u;
        } else {
            for (int64_t w = lane; w < a.bit_words; w += 32) bits[w] = 0u;
        }
        __syncwarp();
    }
}

struct SearchWork {
    DevBuf bits, visits, ldist, flag, entries;
    int64_t bits_bytes = 0;
};
thread_local SearchWork g_search;

}  // namespace

void knn_search_dev(const float* X, int64_t n, int d, const int32_t* gptr, const int32_t* gidx, const int32_t* land,
                    int64_t n_land, const int32_t* entries_host, const float* Q, int64_t m, int k, int ef,
                    int n_entry, int order, int32_t* out_i, float* out_d, cudaStream_t s) {
    if (m == 0) return;
    const size_t smem = sizeof(WarpHeaps) * kSearchWarps;
    static thread_local bool attr = false;
    if (!attr) {
        MGB_CUDA(cudaFuncSetAttribute((const void*)search_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MGB_CUDA(cudaFuncSetAttribute((const void*)search_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MGB_CUDA(cudaFuncSetAttribute((const void*)search_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    int per_sm = 0;
    MGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, search_kernel<0>, 32 * kSearchWarps, smem));
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((m + kSearchWarps - 1) / kSearchWarps,
                                                                  (int64_t)std::max(1, per_sm) * kNumSMs));
    const int64_t slots = blocks * kSearchWarps;
    const int64_t words = (n + 31) / 32;
    SearchWork& w = g_search;
    const int64_t need = slots * words * (int64_t)sizeof(uint32_t);
    if (need > w.bits_bytes || !w.bits.p) {
        w.bits.ensure((size_t)need);
        MGB_CUDA(cudaMemsetAsync(w.bits.p, 0, (size_t)need, s));   // kept zero by every query after
        w.bits_bytes = need;
    }
    w.visits.ensure(sizeof(int32_t) * (size_t)slots * kVisitCap);
    w.ldist.ensure(sizeof(float) * (size_t)std::max<int64_t>(1, slots * n_land));
    int* flag = static_cast<int*>(w.flag.ensure(sizeof(int)));
    MGB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    const int32_t* entries = nullptr;
    if (n_land == 0) {
        int32_t* e = static_cast<int32_t*>(w.entries.ensure(sizeof(int32_t) * (size_t)m * n_entry));
        MGB_CUDA(cudaMemcpyAsync(e, entries_host, sizeof(int32_t) * (size_t)m * n_entry, cudaMemcpyHostToDevice, s));
        entries = e;
    }
    SearchArgs a{X, n, d, gptr, gidx, land, n_land, entries, Q, m, k, ef, n_entry, out_i, out_d,
                 w.bits.as<uint32_t>(), words, w.visits.as<int32_t>(), w.ldist.as<float>(), flag};
    if (order == 0) search_kernel<0><<<(unsigned)blocks, 32 * kSearchWarps, smem, s>>>(a);
    else if (order == 1) search_kernel<1><<<(unsigned)blocks, 32 * kSearchWarps, smem, s>>>(a);
    else search_kernel<2><<<(unsigned)blocks, 32 * kSearchWarps, smem, s>>>(a);
    MGB_LAUNCH_CHECK();
    int h = 0;
    MGB_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    MGB_CUDA(cudaStreamSynchronize(s));
    if (h) throw Error(MG_ERR_NOT_SUPPORTED, std::to_string(h) + " queries needed more than " +
                                                 std::to_string(kCandCap) + " candidates; lower ef");
}

int knn_search_max_ef() { return kMaxEf; }

}  // namespace mgb
