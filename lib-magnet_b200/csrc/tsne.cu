// t-SNE pass on the device.
//  * standalone kernels, one per reference call: tsne_attraction (src/fftrep.cpp:129-177), tsne_step (:225-266),
//    tsne_update (:181-220), bbox_2d (:415-434);
//  * the whole loop of optimize_tsne (magnet/tsne.py:132-214, common path) with every step on the device:
//      bbox + grid choice (magnet/tsne.py:30-46) -> [twiddles, kernel spectra when the grid changed
//      (magnet/tsne.py:48-71)] -> spread -> FFT convolution (+ FP64 Z) -> gather fused with the sparse
//      attraction and the gains/momentum step (+ FP64 mean for the recentring, applied by the next bbox pass).
//    The iteration reads its schedule (exaggeration, momentum) and every size from device memory, so one
//    captured CUDA graph is replayed for all iterations.
#include "tsne.cuh"
#include "interp.cuh"
#include "graph.cuh"
#include <vector>
#include <algorithm>
#include <cstdlib>

namespace mgb {

namespace {

constexpr int kThreads = 256;

int grid_blocks(int64_t work, int per_block, int cap_per_sm = 8) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + per_block - 1) / per_block, (int64_t)cap_per_sm * kNumSMs));
}

// ---------------------------------------------------------------------------------------------- attraction
// T lanes per row, lanes stride over the row's edges, fixed-order shuffle reduction.
template <int T>
__global__ void __launch_bounds__(kThreads) attraction2_kernel(const int32_t* __restrict__ ip,
                                                               const int32_t* __restrict__ ix,
                                                               const float* __restrict__ P,
                                                               const float2* __restrict__ Y, int64_t n, float inv_dof,
                                                               float2* __restrict__ out) {
    const int lg = threadIdx.x % T;
    const unsigned gmask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x & 31) / T * T));
    const int64_t groups = (int64_t)gridDim.x * (blockDim.x / T);
    for (int64_t i = (int64_t)blockIdx.x * (blockDim.x / T) + threadIdx.x / T; i < n; i += groups) {
        const float2 yi = Y[i];
        float ax = 0.f, ay = 0.f;
        const int32_t e1 = ip[i + 1];
        for (int32_t e = ip[i] + lg; e < e1; e += T) {
            const float2 yj = __ldg(&Y[ix[e]]);
            const float dx = yi.x - yj.x, dy = yi.y - yj.y;
            const float w = P[e] / (1.f + (dx * dx + dy * dy) * inv_dof);
            ax += w * dx; ay += w * dy;
        }
#pragma unroll
        for (int o = T / 2; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(gmask, ax, o, T);
            ay += __shfl_xor_sync(gmask, ay, o, T);
        }
        if (lg == 0) out[i] = make_float2(ax, ay);
    }
}

// any dimension (<= 64): one thread per row
__global__ void attractionN_kernel(const int32_t* __restrict__ ip, const int32_t* __restrict__ ix,
                                   const float* __restrict__ P, const float* __restrict__ Y, int64_t n, int dim,
                                   float inv_dof, float* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float acc[kMaxDim];
        for (int d = 0; d < dim; ++d) acc[d] = 0.f;
        const float* yi = Y + i * dim;
        for (int32_t e = ip[i]; e < ip[i + 1]; ++e) {
            const float* yj = Y + (int64_t)ix[e] * dim;
            float d2 = 0.f;
            for (int d = 0; d < dim; ++d) { const float t = yi[d] - yj[d]; d2 += t * t; }
            const float w = P[e] / (1.f + d2 * inv_dof);
            for (int d = 0; d < dim; ++d) acc[d] += w * (yi[d] - yj[d]);
        }
        for (int d = 0; d < dim; ++d) out[i * dim + d] = acc[d];
    }
}

// ---------------------------------------------------------------------------------------------- step
// The gains / momentum / position update of one coordinate, in the reference's evaluation order
// (src/fftrep.cpp:245-253), without contraction into FMAs.
__device__ __forceinline__ float step_coord(float y, float& u, float& gain, float g_, float lr, float momentum) {
    const bool same = (g_ > 0.f) == (u > 0.f);
    float g = same ? __fmul_rn(gain, 0.8f) : __fadd_rn(gain, 0.2f);
    if (g < 0.01f) g = 0.01f;
    gain = g;
    const float un = __fsub_rn(__fmul_rn(momentum, u), __fmul_rn(__fmul_rn(lr, g), g_));
    u = un;
    return __fadd_rn(y, un);
}

// mode 0: grad = rho * A - F * inv_sumQ (tsne_step); mode 1: grad given (tsne_update)
__global__ void step_kernel(float* __restrict__ Y, float* __restrict__ U, float* __restrict__ G,
                            const float* __restrict__ A, const float* __restrict__ F, int64_t total, float rho,
                            float inv_sumQ, float lr, float momentum, int mode) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const float g_ = mode == 0 ? __fsub_rn(__fmul_rn(rho, A[k]), __fmul_rn(F[k], inv_sumQ)) : A[k];
        float u = U[k], gain = G[k];
        Y[k] = step_coord(Y[k], u, gain, g_, lr, momentum);
        U[k] = u; G[k] = gain;
    }
}

// column sums in FP64, one block per dimension, fixed order; then the mean as (float)(sum / n)
__global__ void colmean_kernel(const float* __restrict__ Y, int64_t n, int dim, float* __restrict__ mean) {
    __shared__ double red[kThreads / 32];
    const int d = blockIdx.x;
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += (double)Y[i * dim + d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        mean[d] = (float)(t / (double)n);
    }
}

__global__ void subtract_mean_kernel(float* __restrict__ Y, int64_t total, int dim, const float* __restrict__ mean) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x)
        Y[k] -= mean[k % dim];
}

// ---------------------------------------------------------------------------------------------- bbox
struct BBox { float x0, y0, x1, y1; };

__device__ __forceinline__ BBox bbox_merge(BBox a, BBox b) {
    return BBox{fminf(a.x0, b.x0), fminf(a.y0, b.y0), fmaxf(a.x1, b.x1), fmaxf(a.y1, b.y1)};
}

// partials written by other blocks: read through L2 (not the non-coherent L1)
__device__ __forceinline__ BBox ld_bbox(const BBox* p, unsigned b) {
    const float4 v = __ldcg(reinterpret_cast<const float4*>(p) + b);
    return BBox{v.x, v.y, v.z, v.w};
}

__device__ BBox block_bbox(BBox v) {
    __shared__ BBox red[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        BBox w{__shfl_xor_sync(0xffffffffu, v.x0, o), __shfl_xor_sync(0xffffffffu, v.y0, o),
               __shfl_xor_sync(0xffffffffu, v.x1, o), __shfl_xor_sync(0xffffffffu, v.y1, o)};
        v = bbox_merge(v, w);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = bbox_merge(v, red[w]);
    __syncthreads();
    return v;
}

// the last block of a grid merges the grid's partial boxes, every thread a strided share, then one block reduction
// (one thread walking them in turn took about 40 us for 592 partials at the loads' latency); the box is exact,
// whatever the order; the result is in thread 0
__device__ BBox merge_parts(const BBox* part) {
    BBox t{INFINITY, INFINITY, -INFINITY, -INFINITY};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) t = bbox_merge(t, ld_bbox(part, b));
    return block_bbox(t);
}

__global__ void bbox_kernel(const float2* __restrict__ Y, int64_t n, BBox* __restrict__ part,
                            unsigned* __restrict__ counter, float* __restrict__ out4) {
    __shared__ int is_last;
    BBox v{INFINITY, INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 p = Y[i];
        v = bbox_merge(v, BBox{p.x, p.y, p.x, p.y});
    }
    v = block_bbox(v);
    if (threadIdx.x == 0) { part[blockIdx.x] = v; __threadfence(); is_last = atomicAdd(counter, 1u) == gridDim.x - 1; }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const BBox t = merge_parts(part);
    if (threadIdx.x != 0) return;
    out4[0] = t.x0; out4[1] = t.y0; out4[2] = t.x1; out4[3] = t.y1;
    *counter = 0u;
}

// ---------------------------------------------------------------------------------------------- device loop
// Grid choice of FFTRepulsion2D._grid (magnet/tsne.py:30-46) in FP64 as Python computes it, plus the spectrum
// cache key (n_boxes, round(width, 6)) of _kernels (:51) and the twiddle-table key.
__device__ void choose_grid(GridDesc* g, BBox b, const TsneSched& s, const int* __restrict__ fft_len) {
    const double lo0 = (double)b.x0 - 1e-3, lo1 = (double)b.y0 - 1e-3;
    const double hi0 = (double)b.x1 + 1e-3, hi1 = (double)b.y1 + 1e-3;
    const double span = fmax(hi0 - lo0, hi1 - lo1);
    double nbd = ceil(span / s.box_width);
    nbd = fmin(fmax(nbd, (double)s.min_boxes), (double)s.max_boxes);
    int nb = (int)nbd;
    nb = min(s.max_boxes, (nb + 3) / 4 * 4);
    const double width = ((double)nb * s.box_width >= span) ? s.box_width : fmax(span / (double)nb, 1e-12);
    g->xmin = (float)lo0; g->ymin = (float)lo1;
    g->width = (float)width; g->inv_width = 1.f / g->width;
    g->n_boxes = nb; g->N = nb * s.ni;
    const int M = fft_len[2 * g->N];
    g->M = M; g->Mh = M / 2 + 1;
    const long long kw = llrint(width * 1e6);
    if (nb != g->key_nb || kw != g->key_w) {
        g->spec_dirty = 1; g->key_nb = nb; g->key_w = kw; g->spec_width = width;
    } else {
        g->spec_dirty = 0;
    }
    g->tw_dirty = (M != g->tw_M) ? 1 : 0;
    g->tw_M = M;
}

// recentre (Ycur = Ynext - mean) and bounding box; the last block chooses the grid
__global__ void __launch_bounds__(kThreads) loop_bbox_kernel(const float2* __restrict__ Ynext, float2* __restrict__ Ycur,
                                                             int64_t n, GridDesc* __restrict__ g, BBox* __restrict__ part,
                                                             TsneSched s, const int* __restrict__ fft_len) {
    __shared__ int is_last;
    const bool rc = g->recentre != 0;
    const float mx = g->mean[0], my = g->mean[1];
    BBox v{INFINITY, INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float2 p = Ynext[i];
        if (rc) { p.x = __fsub_rn(p.x, mx); p.y = __fsub_rn(p.y, my); }
        Ycur[i] = p;
        v = bbox_merge(v, BBox{p.x, p.y, p.x, p.y});
    }
    v = block_bbox(v);
    if (threadIdx.x == 0) { part[blockIdx.x] = v; __threadfence(); is_last = atomicAdd(&g->counter2, 1u) == gridDim.x - 1; }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const BBox t = merge_parts(part);
    if (threadIdx.x != 0) return;
    choose_grid(g, t, s, fft_len);
    g->counter2 = 0u;
}

// gather of the potentials + sparse attraction + gains/momentum step for T lanes per point; FP64 column sums of
// the new layout for the recentring (the last block turns them into the mean and advances the iteration)
template <int NI, int T>
__global__ void __launch_bounds__(kThreads) loop_iter_kernel(const float2* __restrict__ Ycur, float2* __restrict__ Ynext,
                                                             float2* __restrict__ U, float2* __restrict__ G,
                                                             const int32_t* __restrict__ ip, const int32_t* __restrict__ ix,
                                                             const float* __restrict__ P, int64_t n,
                                                             GridDesc* __restrict__ gd, const float* __restrict__ phi,
                                                             int pitchP, TsneSched s, double2* __restrict__ mpart) {
    __shared__ double2 red[kThreads / 32];
    __shared__ int is_last;
    const int it = gd->iter;
    const bool early = it < s.early_iter;
    const float rho = early ? s.early_exag : s.exag;
    const float mom = early ? s.mom0 : s.mom1;
    const float inv_sumQ = gd->inv_sumQ;
    const float xmin = gd->xmin, ymin = gd->ymin, width = gd->width, inv_w = gd->inv_width;
    const int nb = gd->n_boxes;
    const size_t plane = (size_t)pitchP * pitchP;
    const int lg = threadIdx.x % T;
    const unsigned gmask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x & 31) / T * T));
    double sx = 0.0, sy = 0.0;
    const int64_t groups = (int64_t)gridDim.x * (blockDim.x / T);
    for (int64_t i = (int64_t)blockIdx.x * (blockDim.x / T) + threadIdx.x / T; i < n; i += groups) {
        const float2 yi = Ycur[i];
        // the gather's loads (which need only y_i) and the step's state are issued first, so that their latency
        // overlaps the attraction's chain of CSR and neighbour loads; the stencil nodes are split over the row's
        // lanes (node q on lane q mod T) and summed by shuffles (src/fftconv.cpp:211-222)
        int bx, by;
        float wx[NI], wy[NI];
        locate<NI>(yi.x, yi.y, xmin, ymin, width, inv_w, nb, bx, by, wx, wy);
        constexpr int kPer = (NI * NI + T - 1) / T;
        float gw[kPer], g1[kPer], g2[kPer], g3[kPer];
#pragma unroll
        for (int r = 0; r < kPer; ++r) {
            const int q = lg + r * T;
            gw[r] = 0.f; g1[r] = 0.f; g2[r] = 0.f; g3[r] = 0.f;
            if (q < NI * NI) {
                const int a = q / NI, b = q - a * NI;
                float wa = 0.f, wb = 0.f;
#pragma unroll
                for (int t = 0; t < NI; ++t) { if (t == a) wa = wx[t]; if (t == b) wb = wy[t]; }
                gw[r] = wa * wb;
                const size_t node = (size_t)(bx * NI + a) * pitchP + (size_t)by * NI + b;
                g1[r] = __ldg(&phi[plane + node]);
                g2[r] = __ldg(&phi[2 * plane + node]);
                g3[r] = __ldg(&phi[3 * plane + node]);
            }
        }
        float2 u = make_float2(0.f, 0.f), gn = make_float2(0.f, 0.f);
        if (lg == 0) { u = U[i]; gn = G[i]; }
        // the row's entries in batches of kBatch per lane: every column index of a batch is read before any
        // neighbour position, so a lane waits for two round trips per batch instead of two per entry (each lane
        // still sums its entries in order)
        constexpr int kBatch = 4;
        float ax = 0.f, ay = 0.f;
        const int32_t e1 = ip[i + 1];
        for (int32_t eb = ip[i] + lg; eb < e1; eb += kBatch * T) {
            int32_t jj[kBatch];
            float pp[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int32_t e = eb + q * T;
                jj[q] = e < e1 ? __ldg(&ix[e]) : -1;
                pp[q] = e < e1 ? __ldg(&P[e]) : 0.f;
            }
            float2 yj[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q) yj[q] = jj[q] >= 0 ? __ldg(&Ycur[jj[q]]) : yi;
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                if (jj[q] >= 0) {
                    const float dx = yi.x - yj[q].x, dy = yi.y - yj[q].y;
                    const float w = pp[q] / (1.f + (dx * dx + dy * dy) * s.inv_dof);
                    ax += w * dx; ay += w * dy;
                }
            }
        }
#pragma unroll
        for (int o = T / 2; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(gmask, ax, o, T);
            ay += __shfl_xor_sync(gmask, ay, o, T);
        }
        float p1 = 0.f, p2 = 0.f, p3 = 0.f;
#pragma unroll
        for (int r = 0; r < kPer; ++r) { p1 += gw[r] * g1[r]; p2 += gw[r] * g2[r]; p3 += gw[r] * g3[r]; }
#pragma unroll
        for (int o = T / 2; o > 0; o >>= 1) {
            p1 += __shfl_xor_sync(gmask, p1, o, T);
            p2 += __shfl_xor_sync(gmask, p2, o, T);
            p3 += __shfl_xor_sync(gmask, p3, o, T);
        }
        if (lg == 0) {
            const float fx = __fsub_rn(__fmul_rn(p1, yi.x), p2), fy = __fsub_rn(__fmul_rn(p1, yi.y), p3);
            const float gx_ = __fsub_rn(__fmul_rn(rho, ax), __fmul_rn(fx, inv_sumQ));
            const float gy_ = __fsub_rn(__fmul_rn(rho, ay), __fmul_rn(fy, inv_sumQ));
            const float nx = step_coord(yi.x, u.x, gn.x, gx_, s.lr, mom);
            const float ny = step_coord(yi.y, u.y, gn.y, gy_, s.lr, mom);
            Ynext[i] = make_float2(nx, ny);
            U[i] = u; G[i] = gn;
            sx += (double)nx; sy += (double)ny;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_double2(sx, sy);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { t.x += red[w].x; t.y += red[w].y; }
        mpart[blockIdx.x] = t;
        __threadfence();
        is_last = atomicAdd(&gd->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // the last block sums the partial sums, every thread a strided share, then a fixed-order block reduction (the
    // same bits from run to run)
    double tx = 0.0, ty = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const double2 v = __ldcg(&mpart[b]);
        tx += v.x; ty += v.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tx += __shfl_xor_sync(0xffffffffu, tx, o);
        ty += __shfl_xor_sync(0xffffffffu, ty, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_double2(tx, ty);
    __syncthreads();
    if (threadIdx.x != 0) return;
    tx = 0.0; ty = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { tx += red[w].x; ty += red[w].y; }
    gd->mean[0] = (float)(tx / (double)n);
    gd->mean[1] = (float)(ty / (double)n);
    gd->recentre = 1;
    gd->iter = it + 1;
    gd->counter = 0u;
}

__global__ void finish_layout_kernel(const float2* __restrict__ Ynext, float2* __restrict__ Yout, int64_t n,
                                     const GridDesc* __restrict__ g) {
    const bool rc = g->recentre != 0;
    const float mx = g->mean[0], my = g->mean[1];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float2 p = Ynext[i];
        if (rc) { p.x = __fsub_rn(p.x, mx); p.y = __fsub_rn(p.y, my); }
        Yout[i] = p;
    }
}

// grad_i += w (Y_i - mean of the partners' positions), one thread per row (src/fftrep.cpp:270-287)
__global__ void mid_spring_kernel(const float* __restrict__ Y, const int32_t* __restrict__ pairs,
                                  float* __restrict__ grad, int64_t n, int dim, int m, float w) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        for (int d = 0; d < dim; ++d) {
            float acc = 0.f;
            for (int k = 0; k < m; ++k) acc += Y[(int64_t)pairs[i * m + k] * dim + d];
            grad[i * dim + d] += w * (Y[i * dim + d] - acc / m);
        }
    }
}

// The hybrid hand-off in two grid-wide passes: FP64 partial sums of every column and of column 0's squares per
// block, the last block turning them into the means and the scale factor target / std(Y[:, 0]); then
// Y = (Y - mean) * factor.
__global__ void __launch_bounds__(kThreads) center_stats_kernel(const float* __restrict__ Y, int64_t n, int dim,
                                                                double target, double* __restrict__ part,
                                                                unsigned* __restrict__ counter, float* __restrict__ out) {
    __shared__ double red[kThreads / 32][kMaxDim + 1];
    __shared__ int is_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 0; d <= dim; ++d) {
        double s = 0.0;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            const double v = (double)Y[i * dim + (d < dim ? d : 0)];
            s += d < dim ? v : v * v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp][d] = s;
    }
    __syncthreads();
    if (threadIdx.x <= dim) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
        part[(size_t)blockIdx.x * (kMaxDim + 1) + threadIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    if (threadIdx.x <= dim) {
        double t = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) t += __ldcg(&part[(size_t)b * (kMaxDim + 1) + threadIdx.x]);
        red[0][threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int d = 0; d < dim; ++d) out[d] = (float)(red[0][d] / (double)n);
        const double m0 = red[0][0] / (double)n;
        const double var = fmax(red[0][dim] / (double)n - m0 * m0, 0.0);
        out[kMaxDim] = (float)(target / fmax(sqrt(var), 1e-12));
        *counter = 0u;
    }
}

__global__ void center_apply_kernel(float* __restrict__ Y, int64_t total, int dim, const float* __restrict__ st) {
    const float f = st[kMaxDim];
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x)
        Y[k] = (Y[k] - st[k % dim]) * f;
}

__global__ void init_opt_state_kernel(float2* U, float2* G, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        U[i] = make_float2(0.f, 0.f);
        G[i] = make_float2(1.f, 1.f);
    }
}

// ---------------------------------------------------------------------------------------------- spatial order
constexpr int kOrderBits = 10;                     // box index bits per axis (n_boxes <= 1000 < 2^10)
constexpr int64_t kOrderBins = 1LL << (2 * kOrderBits);
constexpr int64_t kReorderMinPoints = 20000;       // smaller layouts stay in L1 / L2 whatever their order

__device__ __forceinline__ uint32_t morton_spread(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// the Morton index of each point's box in the last iteration's grid (positions with the pending recentring)
__global__ void order_key_kernel(const float2* __restrict__ Y, int64_t n, const GridDesc* __restrict__ g,
                                 int32_t* __restrict__ key, int32_t* __restrict__ cnt) {
    const bool rc = g->recentre != 0;
    const float mx = g->mean[0], my = g->mean[1];
    const float xmin = g->xmin, ymin = g->ymin, inv_w = g->inv_width;
    const float top = (float)max(g->n_boxes - 1, 0);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float2 p = Y[i];
        if (rc) { p.x -= mx; p.y -= my; }
        const float fx = fminf(fmaxf((p.x - xmin) * inv_w, 0.f), top);   // NaN -> 0
        const float fy = fminf(fmaxf((p.y - ymin) * inv_w, 0.f), top);
        const int32_t k = (int32_t)(morton_spread((uint32_t)fx) | (morton_spread((uint32_t)fy) << 1));
        key[i] = k;
        atomicAdd(&cnt[k], 1);
    }
}

// counting-sort scatter: the new row of point i (cursor = the bin counts, cleared)
__global__ void order_scatter_kernel(const int32_t* __restrict__ key, int64_t n, const int64_t* __restrict__ start,
                                     int32_t* __restrict__ cursor, int32_t* __restrict__ src,
                                     int32_t* __restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = key[i];
        const int64_t r = start[k] + atomicAdd(&cursor[k], 1);
        src[r] = (int32_t)i;
        dst[i] = (int32_t)r;
    }
}

// per-point state into the new order; the new rows' affinity row lengths
__global__ void order_gather_kernel(const int32_t* __restrict__ src, int64_t n, const float2* __restrict__ Y,
                                    const float2* __restrict__ U, const float2* __restrict__ G,
                                    const int32_t* __restrict__ perm, bool permuted, const int32_t* __restrict__ ip,
                                    float2* __restrict__ Yt, float2* __restrict__ Ut, float2* __restrict__ Gt,
                                    int32_t* __restrict__ perm_t, int32_t* __restrict__ len) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t o = src[r];
        Yt[r] = Y[o]; Ut[r] = U[o]; Gt[r] = G[o];
        perm_t[r] = permuted ? perm[o] : o;
        len[r] = ip[o + 1] - ip[o];
    }
}

// one warp per new row: the old row's entries, column indices relabelled
__global__ void order_csr_kernel(const int32_t* __restrict__ src, const int32_t* __restrict__ dst, int64_t n,
                                 const int32_t* __restrict__ ip, const int32_t* __restrict__ ix,
                                 const float* __restrict__ P, const int64_t* __restrict__ newptr,
                                 int32_t* __restrict__ ipt, int32_t* __restrict__ ixt, float* __restrict__ Pt) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
        const int32_t o = src[r];
        const int32_t b = ip[o], e = ip[o + 1];
        const int64_t out = newptr[r];
        for (int32_t j = b + lane; j < e; j += 32) {
            ixt[out + (j - b)] = dst[ix[j]];
            Pt[out + (j - b)] = P[j];
        }
        if (lane == 0) ipt[r] = (int32_t)out;
        if (r == n - 1 && lane == 0) ipt[n] = (int32_t)newptr[n];
    }
}

// the caller's layout into the current row order (Ynext[r] = Y[perm[r]])
__global__ void order_in_kernel(const float2* __restrict__ Yin, const int32_t* __restrict__ perm, int64_t n,
                                float2* __restrict__ Y) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        Y[r] = Yin[perm[r]];
}

// the recentred layout back into the caller's order (Yout[perm[r]] = Ynext[r] - mean)
__global__ void finish_layout_perm_kernel(const float2* __restrict__ Ynext, const int32_t* __restrict__ perm,
                                          float2* __restrict__ Yout, int64_t n, const GridDesc* __restrict__ g) {
    const bool rc = g->recentre != 0;
    const float mx = g->mean[0], my = g->mean[1];
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        float2 p = Ynext[r];
        if (rc) { p.x = __fsub_rn(p.x, mx); p.y = __fsub_rn(p.y, my); }
        Yout[perm[r]] = p;
    }
}

template <int NI, int T>
void launch_iter_t(TsneDev& d, cudaStream_t st) {
    loop_iter_kernel<NI, T><<<d.blocks_iter, kThreads, 0, st>>>(
        d.Ycur.as<float2>(), d.Ynext.as<float2>(), d.U.as<float2>(), d.G.as<float2>(), d.ip.as<int32_t>(),
        d.ix.as<int32_t>(), d.P.as<float>(), d.n, d.g(), d.rb.phi.as<float>(), d.rb.Nmax, d.sch,
        d.mean_part.as<double2>());
}

// resident blocks of the iteration kernel for (NI, T): the grid is one resident wave (the kernel loops over
// rows), so no second partial wave idles the device before the last-block reduction
template <int NI, int T>
int iter_blocks_t() {
    int per_sm = 0;
    MGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, loop_iter_kernel<NI, T>, kThreads, 0));
    return std::max(1, per_sm) * kNumSMs;
}
template <int NI>
int iter_blocks_ni(int tpr) {
    switch (tpr) {
        case 1: return iter_blocks_t<NI, 1>();
        case 2: return iter_blocks_t<NI, 2>();
        case 4: return iter_blocks_t<NI, 4>();
        case 8: return iter_blocks_t<NI, 8>();
        case 16: return iter_blocks_t<NI, 16>();
        default: return iter_blocks_t<NI, 32>();
    }
}

template <int NI>
void launch_iter_ni(TsneDev& d, cudaStream_t st) {
    switch (d.tpr) {
        case 1: launch_iter_t<NI, 1>(d, st); break;
        case 2: launch_iter_t<NI, 2>(d, st); break;
        case 4: launch_iter_t<NI, 4>(d, st); break;
        case 8: launch_iter_t<NI, 8>(d, st); break;
        case 16: launch_iter_t<NI, 16>(d, st); break;
        default: launch_iter_t<NI, 32>(d, st); break;
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------------- standalone API
void tsne_attraction_dev(const int32_t* ip, const int32_t* ix, const float* P, const float* Y, int64_t n, int dim,
                         float dof, float* out, cudaStream_t s) {
    const float inv_dof = 1.f / dof;
    if (n == 0) return;
    if (dim == 2) {
        attraction2_kernel<8><<<grid_blocks(n, kThreads / 8), kThreads, 0, s>>>(
            ip, ix, P, reinterpret_cast<const float2*>(Y), n, inv_dof, reinterpret_cast<float2*>(out));
    } else {
        attractionN_kernel<<<grid_blocks(n, 128), 128, 0, s>>>(ip, ix, P, Y, n, dim, inv_dof, out);
    }
    MGB_LAUNCH_CHECK();
}

static void step_common(float* Y, float* U, float* G, const float* A, const float* F, int64_t n, int dim, float rho,
                        float inv_sumQ, float lr, float momentum, int mode, DevBuf& scratch, cudaStream_t s) {
    const int64_t total = n * dim;
    if (total == 0) return;
    step_kernel<<<grid_blocks(total, kThreads), kThreads, 0, s>>>(Y, U, G, A, F, total, rho, inv_sumQ, lr, momentum,
                                                                  mode);
    MGB_LAUNCH_CHECK();
    float* mean = static_cast<float*>(scratch.ensure(sizeof(float) * kMaxDim));
    colmean_kernel<<<dim, kThreads, 0, s>>>(Y, n, dim, mean);
    MGB_LAUNCH_CHECK();
    subtract_mean_kernel<<<grid_blocks(total, kThreads), kThreads, 0, s>>>(Y, total, dim, mean);
    MGB_LAUNCH_CHECK();
}

void tsne_step_dev(float* Y, float* U, float* G, const float* A, const float* F, int64_t n, int dim, float rho,
                   float inv_sumQ, float lr, float momentum, DevBuf& scratch, cudaStream_t s) {
    step_common(Y, U, G, A, F, n, dim, rho, inv_sumQ, lr, momentum, 0, scratch, s);
}

void tsne_update_dev(float* Y, float* U, float* G, const float* grad, int64_t n, int dim, float lr, float momentum,
                     DevBuf& scratch, cudaStream_t s) {
    step_common(Y, U, G, grad, nullptr, n, dim, 0.f, 0.f, lr, momentum, 1, scratch, s);
}

void mid_spring_dev(const float* Y, const int32_t* pairs, float* grad, int64_t n, int dim, int m, float w,
                    cudaStream_t s) {
    if (n == 0) return;
    mid_spring_kernel<<<grid_blocks(n, kThreads), kThreads, 0, s>>>(Y, pairs, grad, n, dim, m, w);
    MGB_LAUNCH_CHECK();
}

void center_scale_dev(float* Y, int64_t n, int dim, double target_std, DevBuf& scratch, cudaStream_t s) {
    if (n == 0) return;
    const int blocks = grid_blocks(n, kThreads, 4);
    // layout of the scratch: counter at 0, means + factor at 64, per-block partials at 1024
    char* base = static_cast<char*>(scratch.ensure(1024 + sizeof(double) * (kMaxDim + 1) * blocks));
    unsigned* counter = reinterpret_cast<unsigned*>(base);
    float* st = reinterpret_cast<float*>(base + 64);
    double* part = reinterpret_cast<double*>(base + 1024);
    MGB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
    center_stats_kernel<<<blocks, kThreads, 0, s>>>(Y, n, dim, target_std, part, counter, st);
    MGB_LAUNCH_CHECK();
    center_apply_kernel<<<grid_blocks(n * dim, kThreads, 8), kThreads, 0, s>>>(Y, n * dim, dim, st);
    MGB_LAUNCH_CHECK();
}

void bbox_dev(const float* Y, int64_t n, float* out4_dev, DevBuf& scratch, cudaStream_t s) {
    const int blocks = grid_blocks(n, kThreads, 4);
    char* base = static_cast<char*>(scratch.ensure(sizeof(BBox) * blocks + 64));
    unsigned* counter = reinterpret_cast<unsigned*>(base);
    BBox* part = reinterpret_cast<BBox*>(base + 64);
    MGB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
    bbox_kernel<<<blocks, kThreads, 0, s>>>(reinterpret_cast<const float2*>(Y), n, part, counter, out4_dev);
    MGB_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------------------------- TsneDev
TsneDev::~TsneDev() {
    if (graph) cudaGraphExecDestroy(graph);
}

void TsneDev::init(const int32_t* ip_h, const int32_t* ix_h, const float* P_h, int64_t n_, int64_t nnz_, bool host,
                   const TsneSched& s, float dof_, int threads_per_row, cudaStream_t st) {
    require(n_ >= 1, "the layout needs at least one point");
    require(s.ni >= 1 && s.ni <= 8, "n_interp must be between 1 and 8");
    require(s.min_boxes >= 1 && s.max_boxes >= s.min_boxes, "invalid box limits");
    n = n_; nnz = nnz_; ni = s.ni; sch = s; dof = dof_;
    permuted = false;   // the affinities are copied afresh below, in the caller's order
    // MAGNET_TSNE_REORDER_EVERY: iterations between spatial reorders (0, the default, turns them off: sorted
    // points make a warp's spread atomics collide on the same nodes, which costs what the gather gains)
    if (const char* v = std::getenv("MAGNET_TSNE_REORDER_EVERY")) reorder_every = std::max(0, std::atoi(v));
    else reorder_every = 0;
    if (threads_per_row <= 0) {
        const double deg = n > 0 ? (double)nnz / (double)n : 0.0;
        tpr = deg < 3 ? 1 : deg < 6 ? 2 : deg < 12 ? 4 : deg < 40 ? 8 : deg < 100 ? 16 : 32;
    } else {
        tpr = threads_per_row >= 32 ? 32 : threads_per_row >= 16 ? 16 : threads_per_row >= 8 ? 8
            : threads_per_row >= 4 ? 4 : threads_per_row >= 2 ? 2 : 1;
    }
    const cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    Ycur.ensure(sizeof(float2) * n); Ynext.ensure(sizeof(float2) * n);
    U.ensure(sizeof(float2) * n); G.ensure(sizeof(float2) * n);
    ip.ensure(sizeof(int32_t) * (n + 1)); ix.ensure(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
    P.ensure(sizeof(float) * std::max<int64_t>(nnz, 1));
    MGB_CUDA(cudaMemcpyAsync(ip.p, ip_h, sizeof(int32_t) * (n + 1), kind, st));
    if (nnz > 0) {
        MGB_CUDA(cudaMemcpyAsync(ix.p, ix_h, sizeof(int32_t) * nnz, kind, st));
        MGB_CUDA(cudaMemcpyAsync(P.p, P_h, sizeof(float) * nnz, kind, st));
    }
    const int Nmax = s.max_boxes * s.ni;
    rb.alloc(Nmax, next_fft_len(2 * Nmax), s.ni);
    rep_prepare_device_spectra(rb);
    gdesc.ensure(sizeof(GridDesc));
    MGB_CUDA(cudaMemsetAsync(gdesc.p, 0, sizeof(GridDesc), st));
    blocks_bbox = grid_blocks(n, kThreads, 4);
    int resident = 0;
    switch (s.ni) {
        case 1: resident = iter_blocks_ni<1>(tpr); break;
        case 2: resident = iter_blocks_ni<2>(tpr); break;
        case 3: resident = iter_blocks_ni<3>(tpr); break;
        case 4: resident = iter_blocks_ni<4>(tpr); break;
        case 5: resident = iter_blocks_ni<5>(tpr); break;
        case 6: resident = iter_blocks_ni<6>(tpr); break;
        case 7: resident = iter_blocks_ni<7>(tpr); break;
        default: resident = iter_blocks_ni<8>(tpr); break;
    }
    blocks_iter = std::min(grid_blocks(n, kThreads / tpr, 8), resident);
    bbox_part.ensure(sizeof(BBox) * blocks_bbox);
    mean_part.ensure(sizeof(double2) * blocks_iter);
    if (graph && signature() != graph_sig) { cudaGraphExecDestroy(graph); graph = nullptr; }
}

std::string TsneDev::signature() const {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%lld %lld %d %d %g %d %g %g %g %g %g %g %.17g %d %d %d %p %p %p %p %p %p %p %p %p %p %d %d",
                  (long long)n, (long long)nnz, ni, tpr, (double)dof, sch.early_iter, (double)sch.early_exag,
                  (double)sch.exag, (double)sch.mom0, (double)sch.mom1, (double)sch.lr, (double)sch.inv_dof,
                  sch.box_width, sch.min_boxes, sch.max_boxes, sch.ni, Ycur.p, Ynext.p, U.p, G.p, ip.p, ix.p, P.p,
                  gdesc.p, rb.W.p, rb.phi.p, rb.Nmax, rb.Mmax);
    return std::string(buf);
}

void TsneDev::set_layout(const float* Y, bool host, cudaStream_t st) {
    if (permuted) {
        // rows are in the spatial order of the previous run: bring the caller's layout into it
        Yt.ensure(sizeof(float2) * n);
        MGB_CUDA(cudaMemcpyAsync(Yt.p, Y, sizeof(float2) * n, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                 st));
        order_in_kernel<<<grid_blocks(n, kThreads), kThreads, 0, st>>>(Yt.as<float2>(), perm.as<int32_t>(), n,
                                                                          Ynext.as<float2>());
        MGB_LAUNCH_CHECK();
    } else {
        MGB_CUDA(cudaMemcpyAsync(Ynext.p, Y, sizeof(float2) * n, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                 st));
    }
    init_opt_state_kernel<<<grid_blocks(n, kThreads), kThreads, 0, st>>>(U.as<float2>(), G.as<float2>(), n);
    MGB_LAUNCH_CHECK();
    // no pending recentring, iteration 0, empty spectrum and twiddle keys
    GridDesc zero{};
    zero.key_nb = -1; zero.tw_M = -1;
    MGB_CUDA(cudaMemcpyAsync(gdesc.p, &zero, sizeof(GridDesc), cudaMemcpyHostToDevice, st));
    MGB_CUDA(cudaStreamSynchronize(st));   // `zero` lives on this stack frame
}

void TsneDev::get_layout(float* Y, bool host, cudaStream_t st) {
    if (permuted) {
        float2* out = host ? Ycur.as<float2>() : reinterpret_cast<float2*>(Y);
        finish_layout_perm_kernel<<<grid_blocks(n, kThreads), kThreads, 0, st>>>(Ynext.as<float2>(), perm.as<int32_t>(),
                                                                                 out, n, g());
        MGB_LAUNCH_CHECK();
        if (host) {
            MGB_CUDA(cudaMemcpyAsync(Y, Ycur.p, sizeof(float2) * n, cudaMemcpyDeviceToHost, st));
            MGB_CUDA(cudaStreamSynchronize(st));
        }
        return;
    }
    if (host) {
        finish_layout_kernel<<<grid_blocks(n, kThreads), kThreads, 0, st>>>(Ynext.as<float2>(), Ycur.as<float2>(), n, g());
        MGB_LAUNCH_CHECK();
        MGB_CUDA(cudaMemcpyAsync(Y, Ycur.p, sizeof(float2) * n, cudaMemcpyDeviceToHost, st));
        MGB_CUDA(cudaStreamSynchronize(st));
    } else {
        finish_layout_kernel<<<grid_blocks(n, kThreads), kThreads, 0, st>>>(Ynext.as<float2>(), reinterpret_cast<float2*>(Y), n, g());
        MGB_LAUNCH_CHECK();
    }
}

void TsneDev::iterate(cudaStream_t st, cudaEvent_t* ev) {
    auto mark = [&](int k) { if (ev) MGB_CUDA(cudaEventRecord(ev[k], st)); };
    mark(0);
    loop_bbox_kernel<<<blocks_bbox, kThreads, 0, st>>>(Ynext.as<float2>(), Ycur.as<float2>(), n, g(),
                                                      bbox_part.as<BBox>(), sch, rb.fft_len_table.as<int>());
    MGB_LAUNCH_CHECK();
    mark(1);
    rep_twiddles(g(), rb, st, false);
    mark(2);
    rep_update_spectra(g(), rb, dof, st);
    mark(3);
    rep_spread(Ycur.as<float2>(), n, g(), rb, st);
    mark(4);
    rep_convolve(g(), rb, n, st, ev ? ev + 5 : nullptr);
    switch (ni) {
        case 1: launch_iter_ni<1>(*this, st); break;
        case 2: launch_iter_ni<2>(*this, st); break;
        case 3: launch_iter_ni<3>(*this, st); break;
        case 4: launch_iter_ni<4>(*this, st); break;
        case 5: launch_iter_ni<5>(*this, st); break;
        case 6: launch_iter_ni<6>(*this, st); break;
        case 7: launch_iter_ni<7>(*this, st); break;
        default: launch_iter_ni<8>(*this, st); break;
    }
    MGB_LAUNCH_CHECK();
    mark(8);
}

bool TsneDev::reorder_due(int i) const {
    return reorder_every > 0 && n >= kReorderMinPoints && n <= INT32_MAX && i % reorder_every == 1;
}

void TsneDev::reorder(cudaStream_t st) {
    const int blocks = grid_blocks(n, kThreads);
    okey.ensure(sizeof(int32_t) * n);
    ocnt.ensure(sizeof(int32_t) * kOrderBins);
    ostart.ensure(sizeof(int64_t) * (kOrderBins + 1));
    osrc.ensure(sizeof(int32_t) * n); onew.ensure(sizeof(int32_t) * n); olen.ensure(sizeof(int32_t) * n);
    oip.ensure(sizeof(int64_t) * (n + 1));
    Yt.ensure(sizeof(float2) * n); Ut.ensure(sizeof(float2) * n); Gt.ensure(sizeof(float2) * n);
    perm.ensure(sizeof(int32_t) * n); perm_t.ensure(sizeof(int32_t) * n);
    ipt.ensure(sizeof(int32_t) * (n + 1));
    ixt.ensure(sizeof(int32_t) * std::max<int64_t>(nnz, 1)); Pt.ensure(sizeof(float) * std::max<int64_t>(nnz, 1));
    MGB_CUDA(cudaMemsetAsync(ocnt.p, 0, sizeof(int32_t) * kOrderBins, st));
    order_key_kernel<<<blocks, kThreads, 0, st>>>(Ynext.as<float2>(), n, g(), okey.as<int32_t>(), ocnt.as<int32_t>());
    MGB_LAUNCH_CHECK();
    exclusive_scan_i32(ocnt.as<int32_t>(), kOrderBins, ostart.as<int64_t>(), oscan, st);
    MGB_CUDA(cudaMemsetAsync(ocnt.p, 0, sizeof(int32_t) * kOrderBins, st));
    order_scatter_kernel<<<blocks, kThreads, 0, st>>>(okey.as<int32_t>(), n, ostart.as<int64_t>(), ocnt.as<int32_t>(),
                                                      osrc.as<int32_t>(), onew.as<int32_t>());
    MGB_LAUNCH_CHECK();
    order_gather_kernel<<<blocks, kThreads, 0, st>>>(osrc.as<int32_t>(), n, Ynext.as<float2>(), U.as<float2>(),
                                                     G.as<float2>(), perm.as<int32_t>(), permuted, ip.as<int32_t>(),
                                                     Yt.as<float2>(), Ut.as<float2>(), Gt.as<float2>(),
                                                     perm_t.as<int32_t>(), olen.as<int32_t>());
    MGB_LAUNCH_CHECK();
    exclusive_scan_i32(olen.as<int32_t>(), n, oip.as<int64_t>(), oscan, st);
    order_csr_kernel<<<grid_blocks(n * 32, kThreads), kThreads, 0, st>>>(
        osrc.as<int32_t>(), onew.as<int32_t>(), n, ip.as<int32_t>(), ix.as<int32_t>(), P.as<float>(), oip.as<int64_t>(),
        ipt.as<int32_t>(), ixt.as<int32_t>(), Pt.as<float>());
    MGB_LAUNCH_CHECK();
    // back into the buffers the captured iteration reads
    MGB_CUDA(cudaMemcpyAsync(Ynext.p, Yt.p, sizeof(float2) * n, cudaMemcpyDeviceToDevice, st));
    MGB_CUDA(cudaMemcpyAsync(U.p, Ut.p, sizeof(float2) * n, cudaMemcpyDeviceToDevice, st));
    MGB_CUDA(cudaMemcpyAsync(G.p, Gt.p, sizeof(float2) * n, cudaMemcpyDeviceToDevice, st));
    MGB_CUDA(cudaMemcpyAsync(perm.p, perm_t.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    MGB_CUDA(cudaMemcpyAsync(ip.p, ipt.p, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToDevice, st));
    if (nnz > 0) {
        MGB_CUDA(cudaMemcpyAsync(ix.p, ixt.p, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, st));
        MGB_CUDA(cudaMemcpyAsync(P.p, Pt.p, sizeof(float) * nnz, cudaMemcpyDeviceToDevice, st));
    }
    permuted = true;
}

void TsneDev::run(int n_iter, bool use_graph, cudaStream_t st) {
    if (n_iter <= 0) return;
    if (!use_graph) {
        for (int i = 0; i < n_iter; ++i) {
            if (reorder_due(i)) reorder(st);
            iterate(st);
        }
        return;
    }
    if (graph && graph_stream != st) { cudaGraphExecDestroy(graph); graph = nullptr; }
    if (!graph) {
        // capture on a private stream (capture on the legacy default stream is not allowed), replay on st
        cudaStream_t cap;
        MGB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t gr = nullptr;
        try {
            MGB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = launch_count();
            iterate(cap);
            graph_kernels = launch_count() - before;
            MGB_CUDA(cudaStreamEndCapture(cap, &gr));
        } catch (...) {
            cudaGraph_t tmp = nullptr;
            cudaStreamEndCapture(cap, &tmp);
            if (tmp) cudaGraphDestroy(tmp);
            cudaStreamDestroy(cap);
            throw;
        }
        cudaStreamDestroy(cap);
        MGB_CUDA(cudaGraphInstantiate(&graph, gr, 0));
        cudaGraphDestroy(gr);
        graph_stream = st;
        graph_sig = signature();
        count_launch(0 - graph_kernels);   // captured, not run: the replays below count them
    }
    for (int i = 0; i < n_iter; ++i) {
        if (reorder_due(i)) reorder(st);
        MGB_CUDA(cudaGraphLaunch(graph, st));
        count_launch(graph_kernels);
    }
}

void TsneDev::run_profiled(int n_iter, cudaStream_t st, double* stage_ms, int* grid) {
    cudaEvent_t ev[9];
    for (auto& e : ev) MGB_CUDA(cudaEventCreate(&e));
    try {
        for (int it = 0; it < n_iter; ++it) {
            float ro = 0.f;
            if (reorder_due(it)) {   // counted with stage 0 (bbox + grid choice) and in the total
                MGB_CUDA(cudaEventRecord(ev[0], st));
                reorder(st);
                MGB_CUDA(cudaEventRecord(ev[1], st));
                MGB_CUDA(cudaEventSynchronize(ev[1]));
                MGB_CUDA(cudaEventElapsedTime(&ro, ev[0], ev[1]));
                stage_ms[0] += ro;
                stage_ms[8] += ro;
            }
            iterate(st, ev);
            MGB_CUDA(cudaEventSynchronize(ev[8]));
            for (int k = 0; k < 8; ++k) {
                float ms = 0.f;
                MGB_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
                stage_ms[k] += ms;
            }
            float all = 0.f;
            MGB_CUDA(cudaEventElapsedTime(&all, ev[0], ev[8]));
            stage_ms[8] += all;
        }
        GridDesc gh;
        MGB_CUDA(cudaMemcpy(&gh, gdesc.p, sizeof(GridDesc), cudaMemcpyDeviceToHost));
        if (grid) { grid[0] = gh.n_boxes; grid[1] = gh.N; grid[2] = gh.M; grid[3] = gh.Mh; }
    } catch (...) {
        for (auto& e : ev) cudaEventDestroy(e);
        throw;
    }
    for (auto& e : ev) cudaEventDestroy(e);
}

}  // namespace mgb
