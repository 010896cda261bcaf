// The fuzzy neighbour graph on the device.
//
// smooth_knn (src/graph.cpp:29-78): one thread per row. The row's distance sum (FP64) and rho, then the bisection
// of sigma until sum_j exp(-(d_j - rho) / sigma) is within 1e-5 of log2(n_neighbors) * bandwidth, in the
// reference's order of float operations; the floor of sigma at 1e-3 times the row's (or, for rho = 0, the whole
// array's) mean distance; then the memberships. exp is evaluated in FP64 and rounded to float: the reference's
// expf (glibc) agrees with that rounding on all but about 1e-4 of the float inputs, so a bisection decision
// differs only when a sum lands within an ulp of the target and sigma moves by about an ulp.
//
// Fuzzy union (magnet/knn.py:215-230): scipy's csr_matrix((vals, (rows, ind))) sums duplicate columns of a row and
// eliminate_zeros drops zero memberships; T = A^T; P = mix (A + T - A o T) + (1 - mix) (A o T), float32 as scipy
// evaluates it, zeros dropped, columns sorted. On the device:
//   1. each row of A sorted by column (stable), duplicates summed in row order, zeros dropped;
//   2. T by a counting scatter: column counts, an exclusive scan, atomic slots, then each T row sorted by row
//      (one warp per row, a bitonic network in shared memory; heapsort for the rare rows past 512 entries);
//   3. per row, a merge of the sorted A and T rows, counted, scanned into indptr, then written.
// This file is compiled without FMA contraction (-fmad=false), so each product and sum rounds on its own as in
// the reference's x86-64 build and numpy.
#include "graph.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace mgb {

namespace {

constexpr int kThreads = 256;

int grid_for(int64_t work, int per_block = kThreads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + per_block - 1) / per_block, 16LL * kNumSMs));
}

__device__ __forceinline__ float exp_rounded(float x) { return (float)exp((double)x); }

// ---------------------------------------------------------------------------------------------- smooth_knn
__global__ void sigma_kernel(const float* __restrict__ D, int64_t n, int k, float target, int n_iter,
                             float* __restrict__ sigma, float* __restrict__ rho, double* __restrict__ part) {
    __shared__ double red[kThreads / 32];
    double block_sum = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float* d = D + i * k;
        double rowsum = 0.0;
        float r = 0.f;
        bool has = false;
        for (int j = 0; j < k; ++j) {
            rowsum += d[j];
            if (!has && d[j] > 0.f) { r = d[j]; has = true; }
        }
        block_sum += rowsum;
        float lo = 0.f, hi = INFINITY, mid = 1.f, sg = 1.f;
        bool done = false;
        for (int it = 0; it < n_iter; ++it) {
            float psum = 0.f;
            for (int j = 0; j < k; ++j) {
                const float dmr = d[j] - r;
                psum += dmr > 0.f ? exp_rounded(-dmr / mid) : 1.f;
            }
            if (fabsf(psum - target) < 1e-5f) { sg = mid; done = true; break; }
            if (psum > target) { hi = mid; mid = (lo + hi) * 0.5f; }
            else { lo = mid; mid = isinf(hi) ? mid * 2.f : (lo + hi) * 0.5f; }
        }
        if (!done) sg = mid;
        const float mean_row = (float)(rowsum / k);
        if (r > 0.f) sg = fmaxf(sg, 1e-3f * mean_row);
        sigma[i] = sg;
        rho[i] = r;
    }
    // the block's share of the whole array's distance sum
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) block_sum += __shfl_xor_sync(0xffffffffu, block_sum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = block_sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

__global__ void membership_kernel(const float* __restrict__ D, int64_t n, int k, const float* __restrict__ sigma,
                                  const float* __restrict__ rho, const double* __restrict__ part, int n_part,
                                  float* __restrict__ out) {
    __shared__ float mean_all;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < n_part; ++b) t += part[b];
        mean_all = (float)(t / (double)(n * k));
    }
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float r = rho[i];
        float sg = sigma[i];
        if (!(r > 0.f)) sg = fmaxf(sg, 1e-3f * mean_all);
        const float* d = D + i * k;
        float* o = out + i * k;
        for (int j = 0; j < k; ++j) {
            const float dmr = d[j] - r;
            o[j] = dmr > 0.f ? exp_rounded(-dmr / sg) : 1.f;
        }
    }
}

// ---------------------------------------------------------------------------------------------- fuzzy union
// step 1: row i of A into slot i * k: sorted by column (stable insertion sort), duplicates summed in row order,
// zeros dropped; alen[i] = entries kept. Out-of-range columns set *bad.
constexpr int kLocalRow = 32;   // rows up to this length are sorted in a thread-local array

__global__ void a_rows_kernel(const int32_t* __restrict__ ind, const float* __restrict__ vals, int64_t n_rows,
                              int k, int64_t n, int32_t* __restrict__ acol, float* __restrict__ aval,
                              int32_t* __restrict__ alen, int* __restrict__ bad) {
    int32_t lc[kLocalRow];
    float lv[kLocalRow];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_rows; i += (int64_t)gridDim.x * blockDim.x) {
        const bool local = k <= kLocalRow;
        int32_t* c = local ? lc : acol + i * k;
        float* v = local ? lv : aval + i * k;
        for (int j = 0; j < k; ++j) {
            const int32_t col = ind[i * k + j];
            if (col < 0 || col >= n) { atomicExch(bad, 1); alen[i] = 0; return; }
            const float x = vals[i * k + j];
            int p = j;
            while (p > 0 && c[p - 1] > col) { c[p] = c[p - 1]; v[p] = v[p - 1]; --p; }
            c[p] = col; v[p] = x;
        }
        int32_t* oc = acol + i * k;
        float* ov = aval + i * k;
        int m = 0;
        for (int j = 0; j < k;) {
            const int32_t col = c[j];
            float x = v[j];
            int e = j + 1;
            for (; e < k && c[e] == col; ++e) x += v[e];
            if (x != 0.f) { oc[m] = col; ov[m] = x; ++m; }
            j = e;
        }
        alen[i] = m;
    }
}

__global__ void t_count_kernel(const int32_t* __restrict__ acol, const int32_t* __restrict__ alen, int64_t n_rows,
                               int k, int32_t* __restrict__ tcnt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_rows; i += (int64_t)gridDim.x * blockDim.x)
        for (int j = 0; j < alen[i]; ++j) atomicAdd(&tcnt[acol[i * k + j]], 1);
}

__global__ void t_fill_kernel(const int32_t* __restrict__ acol, const float* __restrict__ aval,
                              const int32_t* __restrict__ alen, int64_t n_rows, int k,
                              const int64_t* __restrict__ tptr, int32_t* __restrict__ tcur,
                              int32_t* __restrict__ trow, float* __restrict__ tval) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_rows; i += (int64_t)gridDim.x * blockDim.x)
        for (int j = 0; j < alen[i]; ++j) {
            const int32_t col = acol[i * k + j];
            const int64_t pos = tptr[col] + atomicAdd(&tcur[col], 1);
            trow[pos] = (int32_t)i;
            tval[pos] = aval[i * k + j];
        }
}

__device__ void sift_down(int32_t* key, float* val, int64_t root, int64_t end) {
    while (2 * root + 1 < end) {
        int64_t child = 2 * root + 1;
        if (child + 1 < end && key[child + 1] > key[child]) ++child;
        if (key[root] >= key[child]) return;
        const int32_t tk = key[root]; key[root] = key[child]; key[child] = tk;
        const float tv = val[root]; val[root] = val[child]; val[child] = tv;
        root = child;
    }
}

// step 2b: every T row sorted by row index, one warp per row (the keys of a row are distinct). Rows of up to
// kSortMax entries: a bitonic network over the row padded to a power of two (at least 32) in the warp's own
// shared-memory region; longer rows (hub nodes chosen by very many): heapsort in place by the warp's first lane.
constexpr int kSortWarps = 8;
constexpr int kSortMax = 512;

__global__ void __launch_bounds__(32 * kSortWarps) t_sort_kernel(const int64_t* __restrict__ tptr, int64_t n,
                                                                 int32_t* __restrict__ trow,
                                                                 float* __restrict__ tval) {
    __shared__ int32_t skey[kSortWarps][kSortMax];
    __shared__ float sval[kSortWarps][kSortMax];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int32_t* K = skey[wib];
    float* V = sval[wib];
    const int64_t warps = (int64_t)gridDim.x * kSortWarps;
    for (int64_t r = (int64_t)blockIdx.x * kSortWarps + wib; r < n; r += warps) {
        int32_t* key = trow + tptr[r];
        float* val = tval + tptr[r];
        const int64_t m = tptr[r + 1] - tptr[r];
        if (m <= 1) continue;
        if (m > kSortMax) {
            if (lane == 0) {
                for (int64_t s0 = m / 2 - 1; s0 >= 0; --s0) sift_down(key, val, s0, m);
                for (int64_t e = m - 1; e > 0; --e) {
                    const int32_t tk = key[0]; key[0] = key[e]; key[e] = tk;
                    const float tv = val[0]; val[0] = val[e]; val[e] = tv;
                    sift_down(key, val, 0, e);
                }
            }
            __syncwarp();
            continue;
        }
        int P = 32;
        while (P < m) P <<= 1;
        for (int t = lane; t < P; t += 32) {
            K[t] = t < m ? key[t] : INT32_MAX;
            V[t] = t < m ? val[t] : 0.f;
        }
        __syncwarp();
        for (int k2 = 2; k2 <= P; k2 <<= 1) {
            for (int j = k2 >> 1; j > 0; j >>= 1) {
                for (int t = lane; t < P; t += 32) {
                    const int u = t ^ j;
                    if (u > t) {
                        const bool ascending = (t & k2) == 0;
                        if ((K[t] > K[u]) == ascending) {
                            const int32_t tk = K[t]; K[t] = K[u]; K[u] = tk;
                            const float tv = V[t]; V[t] = V[u]; V[u] = tv;
                        }
                    }
                }
                __syncwarp();
            }
        }
        for (int t = lane; t < m; t += 32) { key[t] = K[t]; val[t] = V[t]; }
        __syncwarp();
    }
}

// P's entry from A's a and T's t (has_a / has_t: present); scipy's float32 order
__device__ __forceinline__ float union_value(bool has_a, float a, bool has_t, float t, float mix, float one_minus_mix) {
    if (has_a && has_t) {
        const float prod = a * t;
        const float d = (a + t) - prod;
        return d * mix + prod * one_minus_mix;
    }
    return (has_a ? a : t) * mix;
}

// step 3: merge A row i and T row i; count (out == nullptr) or write at indptr[i]
template <bool WRITE>
__global__ void union_kernel(const int32_t* __restrict__ acol, const float* __restrict__ aval,
                             const int32_t* __restrict__ alen, int64_t n_rows, int k,
                             const int64_t* __restrict__ tptr, const int32_t* __restrict__ trow,
                             const float* __restrict__ tval, int64_t n, float mix, float one_minus_mix,
                             int32_t* __restrict__ ucnt, const int64_t* __restrict__ uptr,
                             int32_t* __restrict__ indices, float* __restrict__ data) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int la = i < n_rows ? alen[i] : 0;
        const int32_t* ac = acol + i * k;
        const float* av = aval + i * k;
        int64_t ta = tptr[i];
        const int64_t te = tptr[i + 1];
        int ja = 0;
        int64_t out = WRITE ? uptr[i] : 0;
        int cnt = 0;
        while (ja < la || ta < te) {
            const int32_t ca = ja < la ? ac[ja] : INT32_MAX;
            const int32_t ct = ta < te ? trow[ta] : INT32_MAX;
            const int32_t col = ca < ct ? ca : ct;
            const bool has_a = ca == col, has_t = ct == col;
            const float x = union_value(has_a, has_a ? av[ja] : 0.f, has_t, has_t ? tval[ta] : 0.f, mix, one_minus_mix);
            if (has_a) ++ja;
            if (has_t) ++ta;
            if (x != 0.f) {
                if (WRITE) { indices[out] = col; data[out] = x; ++out; }
                ++cnt;
            }
        }
        if (!WRITE) ucnt[i] = cnt;
    }
}

// ---------------------------------------------------------------------------------------------- scan
constexpr int kScanTile = 2048;   // elements per block in the first pass

// per tile: exclusive scan of in[] into out[] (int64) and the tile's total into sums[]
__global__ void __launch_bounds__(1024) scan_tiles_kernel(const int32_t* __restrict__ in, int64_t n,
                                                          int64_t* __restrict__ out, int64_t* __restrict__ sums) {
    __shared__ int64_t sh[1024];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    const int t = threadIdx.x;
    const int64_t i0 = base + 2 * t, i1 = i0 + 1;
    const int64_t x0 = i0 < n ? in[i0] : 0, x1 = i1 < n ? in[i1] : 0;
    sh[t] = x0 + x1;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {   // Hillis-Steele inclusive scan of the pair sums
        const int64_t v = t >= o ? sh[t - o] : 0;
        __syncthreads();
        sh[t] += v;
        __syncthreads();
    }
    const int64_t before = t > 0 ? sh[t - 1] : 0;
    if (i0 < n) out[i0] = before;
    if (i1 < n) out[i1] = before + x0;
    if (t == 1023) sums[blockIdx.x] = sh[1023];
}

// one block: exclusive scan of the tile totals (in place), then the grand total into out[n]
__global__ void __launch_bounds__(1024) scan_sums_kernel(int64_t* __restrict__ sums, int n_tiles,
                                                         int64_t* __restrict__ out, int64_t n) {
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < n_tiles; b0 += 1024) {
        __shared__ int64_t sh[1024];
        const int t = threadIdx.x;
        const int64_t x = b0 + t < n_tiles ? sums[b0 + t] : 0;
        sh[t] = x;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int64_t v = t >= o ? sh[t - o] : 0;
            __syncthreads();
            sh[t] += v;
            __syncthreads();
        }
        if (b0 + t < n_tiles) sums[b0 + t] = carry + sh[t] - x;
        __syncthreads();
        if (t == 0) carry += sh[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

__global__ void scan_add_kernel(int64_t* __restrict__ out, int64_t n, const int64_t* __restrict__ sums) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] += sums[i / kScanTile];
}

// out[0..n] = exclusive scan of in[0..n) and the total
void exclusive_scan(const int32_t* in, int64_t n, int64_t* out, DevBuf& tmp, cudaStream_t s) {
    const int64_t tiles = std::max<int64_t>(1, (n + kScanTile - 1) / kScanTile);
    int64_t* sums = static_cast<int64_t*>(tmp.ensure(sizeof(int64_t) * tiles));
    if (n > 0) {
        scan_tiles_kernel<<<(unsigned)tiles, 1024, 0, s>>>(in, n, out, sums);
        MGB_LAUNCH_CHECK();
    } else {
        MGB_CUDA(cudaMemsetAsync(sums, 0, sizeof(int64_t), s));
    }
    scan_sums_kernel<<<1, 1024, 0, s>>>(sums, (int)tiles, out, n);
    MGB_LAUNCH_CHECK();
    if (n > 0) {
        scan_add_kernel<<<grid_for(n), kThreads, 0, s>>>(out, n, sums);
        MGB_LAUNCH_CHECK();
    }
}

__global__ void narrow_kernel(const int64_t* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)in[i];
}

// ------------------------------------------------------------------------------------------------ transform schedule
// The edge schedule of MAGNET.transform (magnet/__init__.py:907-912) for m new rows of k neighbours, one block:
// freq_i = min(1, s w_i) with s such that sum(freq) = samples_per_node * m (magnet/__init__.py:51-66), the edges with
// freq >= 1 / n_epochs kept in row order with head n_train + row, their neighbour as tail and eps = 1 / freq.
// The reference sorts the weights and walks the breakpoints of the piecewise-linear sum; here s is bracketed by
// bisection in FP64 until the bracket is a few ulps wide, then solved exactly on the segment the bracket lies
// in: s = (target - k) / (sum of the unsaturated weights), k the weights saturated at the bracket. Sums are FP64
// block reductions in a fixed order, so the result is the same from call to call; it differs from the host's
// sorted cumulative sum only by FP64 rounding.
constexpr int kSchedThreads = 1024;

__device__ __forceinline__ double block_sum_d(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    return t;
}

__global__ void __launch_bounds__(kSchedThreads) transform_schedule_kernel(
    const float* __restrict__ w, const int64_t* __restrict__ ind, int64_t n, int k, int64_t n_train, double target,
    double min_freq, int32_t* __restrict__ head, int32_t* __restrict__ tail, float* __restrict__ eps,
    int64_t* __restrict__ n_kept) {
    __shared__ double red[kSchedThreads / 32];
    __shared__ int64_t scan[kSchedThreads / 32];
    __shared__ int64_t carry;
    // sum, positive count, smallest positive weight
    double sum = 0.0, npos = 0.0, wmin = 1e300;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = (double)w[i];
        sum += v;
        if (v > 0.0) { npos += 1.0; wmin = fmin(wmin, v); }
    }
    sum = block_sum_d(sum, red);
    npos = block_sum_d(npos, red);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wmin = fmin(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = wmin;
    __syncthreads();
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) wmin = fmin(wmin, red[i]);
    // s: all ones when n <= target (the reference returns ones, zero weights included); saturating every positive
    // weight when they are too few (the reference's s = 1 / max(w_min, 1e-300)); else the exact solution
    bool ones = (double)n <= target;
    double s = 0.0;
    if (!ones && npos <= target) {
        s = 1e300;
    } else if (!ones) {
        double lo = target / sum, hi = 1.0 / wmin;
        for (int it = 0; it < 200 && hi > lo * (1.0 + 4e-16); ++it) {
            const double mid = 0.5 * (lo + hi);
            double f = 0.0;
            for (int64_t i = threadIdx.x; i < n; i += blockDim.x) f += fmin(1.0, mid * (double)w[i]);
            f = block_sum_d(f, red);
            if (f < target) lo = mid; else hi = mid;
        }
        double cnt = 0.0, rest = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const double v = (double)w[i];
            if (lo * v > 1.0) cnt += 1.0; else rest += v;
        }
        cnt = block_sum_d(cnt, red);
        rest = block_sum_d(rest, red);
        s = rest > 0.0 ? (target - cnt) / rest : hi;
    }
    // the kept edges in row order: a block-wide exclusive scan of the keep flags, 1024 edges at a time
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t base = 0; base < n; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        double freq = 0.0;
        bool keep = false;
        if (i < n) {
            freq = ones ? 1.0 : fmin(1.0, s * (double)w[i]);
            keep = freq >= min_freq;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) scan[warp] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t acc = 0;
            for (int j = 0; j < (int)(blockDim.x >> 5); ++j) { const int64_t t = scan[j]; scan[j] = acc; acc += t; }
            red[0] = (double)acc;   // this tile's count
        }
        __syncthreads();
        if (keep) {
            const int64_t pos = carry + scan[warp] + __popc(bal & ((1u << lane) - 1u));
            head[pos] = (int32_t)(n_train + i / k);
            tail[pos] = (int32_t)ind[i];
            eps[pos] = (float)(1.0 / freq);
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += (int64_t)red[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) *n_kept = carry;
}

// ------------------------------------------------------------------------------------------------ fit schedule
// block partials of the fit schedule's sums over the weights: mode 0: (sum w, count of w > 0, smallest positive
// w); mode 1: (sum of min(1, s w), 0, 0); mode 2: (count of s w > 1, sum of the other w, 0)
constexpr int kSchedBlocks = 4 * kNumSMs;

__global__ void __launch_bounds__(kThreads) sched_sums_kernel(const float* __restrict__ w, int64_t n, int mode,
                                                              double s, double* __restrict__ part) {
    __shared__ double red[3][kThreads / 32];
    double a = 0.0, b = 0.0, c = 1e300;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)w[i];
        if (mode == 0) { a += v; if (v > 0.0) { b += 1.0; c = fmin(c, v); } }
        else if (mode == 1) a += fmin(1.0, s * v);
        else if (s * v > 1.0) b += 1.0;
        else a += v;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c = fmin(c, __shfl_xor_sync(0xffffffffu, c, o));
    }
    if (lane == 0) { red[0][warp] = a; red[1][warp] = b; red[2][warp] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0, tc = 1e300;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { ta += red[0][k]; tb += red[1][k]; tc = fmin(tc, red[2][k]); }
        part[3 * blockIdx.x] = ta;
        part[3 * blockIdx.x + 1] = tb;
        part[3 * blockIdx.x + 2] = tc;
    }
}

__device__ __forceinline__ double sched_freq(double v, double s, bool ones) { return ones ? 1.0 : fmin(1.0, s * v); }

__global__ void sched_flag_kernel(const float* __restrict__ w, int64_t n, double s, bool ones, double min_freq,
                                  int32_t* __restrict__ flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = sched_freq((double)w[i], s, ones) >= min_freq ? 1 : 0;
}

// one thread per row: its kept entries, in order, at their scanned offsets
__global__ void sched_scatter_kernel(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                     const float* __restrict__ w, int64_t n_rows, double s, bool ones,
                                     double min_freq, const int64_t* __restrict__ off, int32_t* __restrict__ head,
                                     int32_t* __restrict__ tail, float* __restrict__ eps) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
        for (int32_t e = indptr[r]; e < indptr[r + 1]; ++e) {
            const double f = sched_freq((double)w[e], s, ones);
            if (f >= min_freq) {
                const int64_t pos = off[e];
                head[pos] = (int32_t)r;
                tail[pos] = indices[e];
                eps[pos] = (float)(1.0 / f);
            }
        }
    }
}

}  // namespace

void exclusive_scan_i32(const int32_t* in, int64_t n, int64_t* out, DevBuf& tmp, cudaStream_t s) {
    exclusive_scan(in, n, out, tmp, s);
}

void smooth_knn_dev(const float* dist, int64_t n_rows, int k, float target, int n_iter, float* out, GraphWork& w,
                    cudaStream_t s) {
    if (n_rows == 0 || k == 0) return;
    float* sigma = static_cast<float*>(w.sigma.ensure(sizeof(float) * n_rows));
    float* rho = static_cast<float*>(w.rho.ensure(sizeof(float) * n_rows));
    const int blocks = grid_for(n_rows);
    double* part = static_cast<double*>(w.part.ensure(sizeof(double) * blocks));
    sigma_kernel<<<blocks, kThreads, 0, s>>>(dist, n_rows, k, target, n_iter, sigma, rho, part);
    MGB_LAUNCH_CHECK();
    membership_kernel<<<blocks, kThreads, 0, s>>>(dist, n_rows, k, sigma, rho, part, blocks, out);
    MGB_LAUNCH_CHECK();
}

int64_t fuzzy_union_dev(const int32_t* ind, const float* vals, int64_t n_rows, int k, int64_t n, float mix,
                        float one_minus_mix, int32_t* indptr, int32_t* indices, float* data, int64_t cap,
                        GraphWork& w, cudaStream_t s) {
    const int64_t ek = std::max<int64_t>(n_rows * k, 1);
    int32_t* acol = static_cast<int32_t*>(w.acol.ensure(sizeof(int32_t) * ek));
    float* aval = static_cast<float*>(w.aval.ensure(sizeof(float) * ek));
    int32_t* alen = static_cast<int32_t*>(w.alen.ensure(sizeof(int32_t) * std::max<int64_t>(n_rows, 1)));
    int32_t* tcnt = static_cast<int32_t*>(w.tcnt.ensure(sizeof(int32_t) * std::max<int64_t>(n, 1)));
    int32_t* tcur = static_cast<int32_t*>(w.tcur.ensure(sizeof(int32_t) * std::max<int64_t>(n, 1)));
    int64_t* tptr = static_cast<int64_t*>(w.tptr.ensure(sizeof(int64_t) * (n + 1)));
    int32_t* trow = static_cast<int32_t*>(w.trow.ensure(sizeof(int32_t) * ek));
    float* tval = static_cast<float*>(w.tval.ensure(sizeof(float) * ek));
    int32_t* ucnt = static_cast<int32_t*>(w.ucnt.ensure(sizeof(int32_t) * std::max<int64_t>(n, 1)));
    int* bad = static_cast<int*>(w.flag.ensure(sizeof(int)));
    int64_t* uptr = static_cast<int64_t*>(w.uptr.ensure(sizeof(int64_t) * (n + 1)));
    MGB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    MGB_CUDA(cudaMemsetAsync(tcnt, 0, sizeof(int32_t) * std::max<int64_t>(n, 1), s));
    MGB_CUDA(cudaMemsetAsync(tcur, 0, sizeof(int32_t) * std::max<int64_t>(n, 1), s));
    if (n_rows > 0 && k > 0) {
        a_rows_kernel<<<grid_for(n_rows), kThreads, 0, s>>>(ind, vals, n_rows, k, n, acol, aval, alen, bad);
        MGB_LAUNCH_CHECK();
        int h_bad = 0;
        MGB_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        MGB_CUDA(cudaStreamSynchronize(s));
        require(h_bad == 0, "neighbour index out of range");
        t_count_kernel<<<grid_for(n_rows), kThreads, 0, s>>>(acol, alen, n_rows, k, tcnt);
        MGB_LAUNCH_CHECK();
    } else {
        MGB_CUDA(cudaMemsetAsync(alen, 0, sizeof(int32_t) * std::max<int64_t>(n_rows, 1), s));
    }
    exclusive_scan(tcnt, n, tptr, w.scan, s);
    if (n_rows > 0 && k > 0) {
        t_fill_kernel<<<grid_for(n_rows), kThreads, 0, s>>>(acol, aval, alen, n_rows, k, tptr, tcur, trow, tval);
        MGB_LAUNCH_CHECK();
    }
    if (n > 0) {
        t_sort_kernel<<<(int)std::min<int64_t>((n + kSortWarps - 1) / kSortWarps, 32LL * kNumSMs),
                        32 * kSortWarps, 0, s>>>(tptr, n, trow, tval);
        MGB_LAUNCH_CHECK();
        union_kernel<false><<<grid_for(n), kThreads, 0, s>>>(acol, aval, alen, n_rows, k, tptr, trow, tval, n, mix,
                                                             one_minus_mix, ucnt, nullptr, nullptr, nullptr);
        MGB_LAUNCH_CHECK();
    }
    exclusive_scan(ucnt, n, uptr, w.scan, s);
    int64_t nnz = 0;
    MGB_CUDA(cudaMemcpyAsync(&nnz, uptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    MGB_CUDA(cudaStreamSynchronize(s));
    require(nnz <= cap, "output capacity too small for the union");
    require(nnz <= INT32_MAX, "the union has more than 2^31 - 1 entries");
    if (n > 0) {
        union_kernel<true><<<grid_for(n), kThreads, 0, s>>>(acol, aval, alen, n_rows, k, tptr, trow, tval, n, mix,
                                                            one_minus_mix, nullptr, uptr, indices, data);
        MGB_LAUNCH_CHECK();
    }
    narrow_kernel<<<grid_for(n + 1), kThreads, 0, s>>>(uptr, n + 1, indptr);
    MGB_LAUNCH_CHECK();
    MGB_CUDA(cudaStreamSynchronize(s));
    return nnz;
}

int64_t transform_schedule_dev(const float* w, const int64_t* ind, int64_t m, int k, int64_t n_train,
                               double samples_per_node, int n_epochs, int32_t* head, int32_t* tail, float* eps,
                               GraphWork& gw, cudaStream_t s) {
    const int64_t n = m * (int64_t)k;
    int64_t* cnt = static_cast<int64_t*>(gw.sched.ensure(sizeof(int64_t)));
    transform_schedule_kernel<<<1, kSchedThreads, 0, s>>>(w, ind, n, k, n_train, samples_per_node * (double)m,
                                                          1.0 / (double)n_epochs, head, tail, eps, cnt);
    MGB_LAUNCH_CHECK();
    int64_t kept = 0;
    MGB_CUDA(cudaMemcpyAsync(&kept, cnt, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    MGB_CUDA(cudaStreamSynchronize(s));
    return kept;
}

namespace {
// the three sums of sched_sums_kernel over the grid, its partials added on the host in block order
void sched_sums(const float* w, int64_t n, int mode, double sc, GraphWork& gw, cudaStream_t s, double out[3]) {
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, kSchedBlocks));
    double* part = static_cast<double*>(gw.s_part.ensure(sizeof(double) * 3 * kSchedBlocks));
    sched_sums_kernel<<<blocks, kThreads, 0, s>>>(w, n, mode, sc, part);
    MGB_LAUNCH_CHECK();
    std::vector<double> h((size_t)3 * blocks);
    MGB_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
    MGB_CUDA(cudaStreamSynchronize(s));
    out[0] = 0.0; out[1] = 0.0; out[2] = 1e300;
    for (int b = 0; b < blocks; ++b) {
        out[0] += h[3 * b];
        out[1] += h[3 * b + 1];
        out[2] = std::min(out[2], h[3 * b + 2]);
    }
}
}  // namespace

int64_t edge_schedule_dev(const int32_t* indptr, const int32_t* indices, const float* w, int64_t n, int64_t nnz,
                          double samples_per_node, int n_epochs, int32_t* head, int32_t* tail, float* eps,
                          GraphWork& gw, cudaStream_t s) {
    if (nnz <= 0) return 0;
    const double target = samples_per_node * (double)n;
    double st[3];
    sched_sums(w, nnz, 0, 0.0, gw, s, st);
    const double sum = st[0], npos = st[1], wmin = st[2];
    // the solution of _sampling_frequencies (magnet/__init__.py:51-66): all ones when nnz <= target; every
    // positive weight saturated when they are too few (the reference's s = 1 / max(w_min, 1e-300)); else s exact
    const bool ones = (double)nnz <= target;
    double sc = 0.0;
    if (!ones && npos <= target) {
        sc = 1e300;
    } else if (!ones) {
        double lo = target / sum, hi = 1.0 / wmin;
        for (int it = 0; it < 200 && hi > lo * (1.0 + 4e-16); ++it) {
            const double mid = 0.5 * (lo + hi);
            double f[3];
            sched_sums(w, nnz, 1, mid, gw, s, f);
            if (f[0] < target) lo = mid; else hi = mid;
        }
        double cr[3];
        sched_sums(w, nnz, 2, lo, gw, s, cr);
        sc = cr[0] > 0.0 ? (target - cr[1]) / cr[0] : hi;
    }
    const double min_freq = 1.0 / (double)n_epochs;
    int32_t* flag = static_cast<int32_t*>(gw.s_flag.ensure(sizeof(int32_t) * (size_t)nnz));
    int64_t* off = static_cast<int64_t*>(gw.s_off.ensure(sizeof(int64_t) * (size_t)(nnz + 1)));
    const int eb = (int)std::max<int64_t>(1, std::min<int64_t>((nnz + kThreads - 1) / kThreads, 16 * kNumSMs));
    sched_flag_kernel<<<eb, kThreads, 0, s>>>(w, nnz, sc, ones, min_freq, flag);
    MGB_LAUNCH_CHECK();
    exclusive_scan_i32(flag, nnz, off, gw.s_tmp, s);
    const int rb = (int)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, 16 * kNumSMs));
    sched_scatter_kernel<<<rb, kThreads, 0, s>>>(indptr, indices, w, n, sc, ones, min_freq, off, head, tail, eps);
    MGB_LAUNCH_CHECK();
    int64_t kept = 0;
    MGB_CUDA(cudaMemcpyAsync(&kept, off + nnz, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    MGB_CUDA(cudaStreamSynchronize(s));
    return kept;
}

}  // namespace mgb
