// FFT-interpolated repulsion on the device: spread, FFT convolution with the kernel spectra, gather.
// Reference: class FFTConv2D::compute, src/fftconv.cpp:58-230 (spread :98-122, FFTs and products :124-199,
// gather :200-229), and FFTRepulsion2D._grid / _kernels, magnet/tsne.py:30-71.
//
// The 2-D transform is rows then columns, as the reference's r2c/c2c pair, but with one complex FFT of
// length M carrying two real rows (two-for-one packing) and the row spectra stored transposed so that the
// column pass reads contiguous columns. The column pass fuses forward transform, product with the real kernel
// spectrum and inverse transform for each output channel, and accumulates Z = sum_k K1h |W0h|^2 / M^2 (the
// same sum as the reference's sum over points of the interpolated potential 0, by Parseval).
#include "fftrep.cuh"
#include "fft3.cuh"
#include "fft.cuh"
#include "interp.cuh"
#include <vector>
#include <cmath>

namespace mgb {

int next_5smooth(int target) {
    if (target <= 1) return 1;
    for (int x = target;; ++x)
        if (fft::is_5smooth(x)) return x;
}

// Any M >= 2N - 1 gives the same circular convolution of the N live nodes (the kernel is sampled at every offset
// in (-N, N) on the M torus), so the device loop may skip the few 5-smooth lengths the in-place engine has no
// plan for (5^5 = 3125 and its multiples need five stages) and take the next one.
int next_fft_len(int target) {
    for (int x = next_5smooth(target);; x = next_5smooth(x + 1)) {
        fft3::Plan p;
        if (x > fft::kMaxLen || fft3::make_plan(x, p)) return x;
    }
}

void ensure_fft_attrs();

void RepBuffers::alloc(int Nmax_, int Mmax_, int ni_) {
    ensure_fft_attrs();
    require(Mmax_ <= fft::kMaxLen, "FFT side " + std::to_string(Mmax_) + " exceeds the supported maximum " +
                                       std::to_string(fft::kMaxLen));
    const bool grow = Nmax_ > Nmax || Mmax_ > Mmax;
    ni = ni_;
    if (!grow) return;
    Nmax = std::max(Nmax, Nmax_);
    Mmax = std::max(Mmax, Mmax_);
    Mhmax = Mmax / 2 + 1;
    Npmax = (Nmax + 3) & ~3;   // transposed spectra of 4 rows at once: 32-byte aligned groups
    W.ensure((size_t)Nmax * Nmax * sizeof(float4));
    MGB_CUDA(cudaMemset(W.p, 0, (size_t)Nmax * Nmax * sizeof(float4)));
    WhT.ensure((size_t)3 * Mhmax * Npmax * sizeof(float2));
    PhT.ensure((size_t)4 * Mhmax * Npmax * sizeof(float2));
    phi.ensure((size_t)4 * Nmax * Nmax * sizeof(float));
    Kt.ensure((size_t)2 * Mhmax * Mmax * sizeof(float));
    tw.ensure((size_t)Mmax * sizeof(float2));
    zpart.ensure((size_t)Mhmax * sizeof(double));
    // The in-place engine runs when the largest length has a plan: an FFTConv2D object computes at M = Mmax only,
    // and the device loop takes its lengths from the table below, which then holds planned lengths only.
    fft3::Plan pmax;
    use3 = fft3::make_plan(Mmax, pmax);
    fft3_build_plans(plans3, Mmax, Mp3max);
    if (use3) fft3_prepare(Mp3max);
    std::vector<int> table(2 * (size_t)Nmax + 2);
    int cur = 1;
    for (size_t t = 0; t < table.size(); ++t) {
        if ((int)t > cur || t == 0) {
            const int target = (int)std::max<size_t>(t, 1);
            cur = use3 ? next_fft_len(target) : next_5smooth(target);
        }
        table[t] = cur;
    }
    fft_len_table.ensure(table.size() * sizeof(int));
    MGB_CUDA(cudaMemcpy(fft_len_table.p, table.data(), table.size() * sizeof(int), cudaMemcpyHostToDevice));
}

namespace {

constexpr int kFftThreads = 512;

struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

__device__ __forceinline__ float chan(const float4& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// ------------------------------------------------------------------------------------------------ spread
// One thread per point, nodes accumulated with vector float atomics. Warps whose 32 points share one box (the
// dense case: early-exaggeration layouts put everything in a few boxes) first reduce the node values with
// shuffles, so one atomic per node replaces 32.
template <int NI>
__global__ void __launch_bounds__(256) spread_kernel(const float2* __restrict__ Y, int64_t n,
                                                     const GridDesc* __restrict__ gd, float4* __restrict__ W,
                                                     int pitch) {
    const float xmin = gd->xmin, ymin = gd->ymin, width = gd->width, inv_w = gd->inv_width;
    const int nb = gd->n_boxes;
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int64_t i = base + lane;
        const bool act = i < n;
        float x = 0.f, y = 0.f;
        if (act) { const float2 p = Y[i]; x = p.x; y = p.y; }
        int bx = 0, by = 0;
        float wx[NI], wy[NI];
        locate<NI>(x, y, xmin, ymin, width, inv_w, nb, bx, by, wx, wy);
        const int key = act ? bx * nb + by : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        if (peers == 0xffffffffu && key >= 0) {
            // whole warp in one box: reduce per node, lane q issues node q
#pragma unroll
            for (int a = 0; a < NI; ++a) {
#pragma unroll
                for (int b = 0; b < NI; ++b) {
                    const float w = wx[a] * wy[b];
                    float s0 = w, s1 = w * x, s2 = w * y;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                    }
                    if (lane == ((a * NI + b) & 31)) {
                        const int gx = bx * NI + a, gy = by * NI + b;
                        atomicAdd(&W[(size_t)gx * pitch + gy], make_float4(s0, s1, s2, 0.f));
                    }
                }
            }
        } else if (act) {
#pragma unroll
            for (int a = 0; a < NI; ++a) {
                const int gx = bx * NI + a;
#pragma unroll
                for (int b = 0; b < NI; ++b) {
                    const int gy = by * NI + b;
                    const float w = wx[a] * wy[b];
                    atomicAdd(&W[(size_t)gx * pitch + gy], make_float4(w, w * x, w * y, 0.f));
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------ rows
// Forward row transforms of the 3 charge channels: rows g0 = 2p and g1 = 2p + 1 packed as one complex
// sequence (z = w_g0 + i w_g1, zero padded to M), transformed, separated, written transposed. Zeroes the W
// rows it consumed so the next spread starts from an empty grid.
__global__ void __launch_bounds__(kFftThreads) row_fwd_kernel(const GridDesc* __restrict__ gd, float4* __restrict__ W,
                                                               int pitchW, float2* __restrict__ WhT, int Np, int Mhmax,
                                                               const float2* __restrict__ tw) {
    extern __shared__ float2 sm[];
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    fft::Plan plan;
    fft::make_plan(M, plan);
    float2* A = sm;
    float2* B = sm + M;
    const int npairs = (N + 1) / 2;
    for (int rp = blockIdx.x; rp < npairs; rp += gridDim.x) {
        const int g0 = 2 * rp, g1 = 2 * rp + 1;
        const bool has1 = g1 < N;
        for (int c = 0; c < 3; ++c) {
            for (int b = threadIdx.x; b < M; b += blockDim.x) {
                float2 z = make_float2(0.f, 0.f);
                if (b < N) {
                    z.x = chan(W[(size_t)g0 * pitchW + b], c);
                    if (has1) z.y = chan(W[(size_t)g1 * pitchW + b], c);
                }
                A[b] = z;
            }
            __syncthreads();
            const float2* R = fft::forward(A, B, plan, tw, threadIdx.x, blockDim.x, BlockSync());
            for (int k = threadIdx.x; k < Mh; k += blockDim.x) {
                const float2 zk = R[k], zm = R[k == 0 ? 0 : M - k];
                // row g0: (Z_k + conj Z_{-k}) / 2 ; row g1: (Z_k - conj Z_{-k}) / 2i
                const float4 v = make_float4(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y),
                                             0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
                *reinterpret_cast<float4*>(WhT + ((size_t)c * Mhmax + k) * Np + g0) = v;
            }
            __syncthreads();
        }
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int b = threadIdx.x; b < N; b += blockDim.x) {
            W[(size_t)g0 * pitchW + b] = z4;
            if (has1) W[(size_t)g1 * pitchW + b] = z4;
        }
    }
}

// Inverse row transforms of the 4 potential channels: rows g0, g1 rebuilt from their half spectra (Hermitian
// extension; DC and Nyquist imaginary parts dropped as a c2r does), one complex inverse FFT for both rows,
// scaled by 1/M^2 (src/fftconv.cpp:176, 188-198).
__global__ void __launch_bounds__(kFftThreads) row_inv_kernel(const GridDesc* __restrict__ gd,
                                                               const float2* __restrict__ PhT, int Np, int Mhmax,
                                                               float* __restrict__ phi, int pitchP,
                                                               const float2* __restrict__ tw) {
    extern __shared__ float2 sm[];
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    fft::Plan plan;
    fft::make_plan(M, plan);
    float2* A = sm;
    float2* B = sm + M;
    const float scale = 1.f / ((float)M * (float)M);
    const bool even = (M & 1) == 0;
    const int npairs = (N + 1) / 2;
    const size_t plane = (size_t)pitchP * pitchP;
    for (int rp = blockIdx.x; rp < npairs; rp += gridDim.x) {
        const int g0 = 2 * rp, g1 = 2 * rp + 1;
        const bool has1 = g1 < N;
        for (int c = 0; c < 4; ++c) {
            for (int k = threadIdx.x; k < M; k += blockDim.x) {
                const int kk = k < Mh ? k : M - k;
                float4 v = *reinterpret_cast<const float4*>(PhT + ((size_t)c * Mhmax + kk) * Np + g0);
                float2 a = make_float2(v.x, v.y), b = make_float2(v.z, v.w);
                if (kk == 0 || (even && kk == M / 2)) { a.y = 0.f; b.y = 0.f; }
                if (k >= Mh) { a.y = -a.y; b.y = -b.y; }
                // Z = a + i b; inverse through the forward transform: conj in, conj out
                A[k] = make_float2(a.x - b.y, -(a.y + b.x));
            }
            __syncthreads();
            const float2* R = fft::forward(A, B, plan, tw, threadIdx.x, blockDim.x, BlockSync());
            for (int b = threadIdx.x; b < N; b += blockDim.x) {
                const float2 z = R[b];   // conj(z) = (z.x, -z.y): row g0 = Re, row g1 = Im
                phi[c * plane + (size_t)g0 * pitchP + b] = z.x * scale;
                if (has1) phi[c * plane + (size_t)g1 * pitchP + b] = -z.y * scale;
            }
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------------------------------------ columns
// Per column k of the row spectra: for each output channel (0: K1 x W0, 1: K2 x W0, 2: K2 x W1, 3: K2 x W2,
// src/fftconv.cpp:157-173), forward column FFT, product with the real kernel spectrum, inverse column FFT,
// keep the N live outputs. Channel 0 also contributes sum_k1 K1h |W0h|^2 to Z. The last block to finish
// reduces the per-column partial sums in a fixed order (deterministic) into sumQ.
__global__ void __launch_bounds__(kFftThreads) col_kernel(GridDesc* __restrict__ gd, const float2* __restrict__ WhT,
                                                           float2* __restrict__ PhT, int Np, int Mhmax,
                                                           const float* __restrict__ Kt, int Mmax,
                                                           const float2* __restrict__ tw,
                                                           double* __restrict__ zpart, int64_t n_points) {
    extern __shared__ float2 sm[];
    __shared__ double red[kFftThreads / 32];
    __shared__ int is_last;
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    fft::Plan plan;
    fft::make_plan(M, plan);
    float2* A = sm;
    float2* B = sm + M;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < Mh; k += gridDim.x) {
        for (int out = 0; out < 4; ++out) {
            const int c = out <= 1 ? 0 : out - 1;
            const float* K = Kt + ((size_t)(out == 0 ? 0 : 1) * Mhmax + k) * Mmax;
            const float2* src = WhT + ((size_t)c * Mhmax + k) * Np;
            for (int a = threadIdx.x; a < M; a += blockDim.x) A[a] = a < N ? src[a] : make_float2(0.f, 0.f);
            __syncthreads();
            float2* R = fft::forward(A, B, plan, tw, threadIdx.x, blockDim.x, BlockSync());
            float2* O = (R == A) ? B : A;
            double zs = 0.0;
            for (int a = threadIdx.x; a < M; a += blockDim.x) {
                const float kv = __ldg(&K[a]);
                const float2 r = R[a];
                if (out == 0) zs += (double)kv * ((double)r.x * r.x + (double)r.y * r.y);
                R[a] = make_float2(r.x * kv, -(r.y * kv));   // conj(K r): inverse through the forward transform
            }
            if (out == 0) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) zs += __shfl_xor_sync(0xffffffffu, zs, o);
                if (lane == 0) red[warp] = zs;
            }
            __syncthreads();
            if (out == 0 && threadIdx.x == 0) {
                double t = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
                const bool single = (k == 0) || ((M & 1) == 0 && k == M / 2);
                zpart[k] = single ? t : 2.0 * t;
            }
            const float2* Q = fft::forward(R, O, plan, tw, threadIdx.x, blockDim.x, BlockSync());
            float2* dst = PhT + ((size_t)out * Mhmax + k) * Np;
            for (int a = threadIdx.x; a < N; a += blockDim.x) { const float2 q = Q[a]; dst[a] = make_float2(q.x, -q.y); }
            __syncthreads();
        }
    }
    // last block: Z = sum of the partials / M^2 - n
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(&gd->counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double t = 0.0;
    for (int k = threadIdx.x; k < Mh; k += blockDim.x) t += __ldcg(&zpart[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        const double sumQ = s / ((double)M * (double)M) - (double)n_points;
        gd->sumQ = sumQ;
        const float sf = (float)sumQ;
        gd->sumQ_f = sf;
        gd->inv_sumQ = (float)(1.0 / fmax((double)sf, 1e-12));
        gd->counter = 0u;
    }
}

// ------------------------------------------------------------------------------------------------ gather
template <int NI>
__global__ void __launch_bounds__(256) gather_forces_kernel(const float2* __restrict__ Y, int64_t n,
                                                            const GridDesc* __restrict__ gd,
                                                            const float* __restrict__ phi, int pitchP,
                                                            float2* __restrict__ F) {
    const float xmin = gd->xmin, ymin = gd->ymin, width = gd->width, inv_w = gd->inv_width;
    const int nb = gd->n_boxes;
    const size_t plane = (size_t)pitchP * pitchP;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 p = Y[i];
        int bx, by;
        float wx[NI], wy[NI];
        locate<NI>(p.x, p.y, xmin, ymin, width, inv_w, nb, bx, by, wx, wy);
        float p1 = 0.f, p2 = 0.f, p3 = 0.f;
#pragma unroll
        for (int a = 0; a < NI; ++a) {
            const size_t row = (size_t)(bx * NI + a) * pitchP + (size_t)by * NI;
#pragma unroll
            for (int b = 0; b < NI; ++b) {
                const float w = wx[a] * wy[b];
                p1 = __fadd_rn(p1, __fmul_rn(w, __ldg(&phi[plane + row + b])));
                p2 = __fadd_rn(p2, __fmul_rn(w, __ldg(&phi[2 * plane + row + b])));
                p3 = __fadd_rn(p3, __fmul_rn(w, __ldg(&phi[3 * plane + row + b])));
            }
        }
        F[i] = make_float2(__fsub_rn(__fmul_rn(p1, p.x), p2), __fsub_rn(__fmul_rn(p1, p.y), p3));
    }
}

// ------------------------------------------------------------------------------------------------ spectra
// exp(-2 pi i m / M) in FP64, rounded once; skipped unless the grid choice flagged a new M (or forced)
__global__ void twiddle_kernel(const GridDesc* __restrict__ gd, float2* __restrict__ tw, int force) {
    if (!force && !gd->tw_dirty) return;
    const int M = gd->M;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)m / (double)M, &s, &c);
        tw[m] = make_float2((float)c, (float)s);
    }
}

// Row spectra of the two kernels (rows a in [0, M/2], the kernels being even in a): z_b = K1(a,b) + i K2(a,b)
// on the wrapped offsets of magnet/tsne.py:57-67, one complex FFT, separated; stored transposed.
__global__ void __launch_bounds__(kFftThreads) spec_rows_kernel(const GridDesc* __restrict__ gd,
                                                                 float2* __restrict__ Rt, int Pa, int Mhmax,
                                                                 const float2* __restrict__ tw, int ni, double dof) {
    if (!gd->spec_dirty) return;
    const double width_d = gd->spec_width;
    extern __shared__ float2 sm[];
    const int M = gd->M, Mh = gd->Mh;
    fft::Plan plan;
    fft::make_plan(M, plan);
    float2* A = sm;
    float2* B = sm + M;
    const double delta = width_d / (double)ni;
    const int nrows = M / 2 + 1;
    for (int a = blockIdx.x; a < nrows; a += gridDim.x) {
        const double oa = (double)(a <= M / 2 ? a : a - M) * delta;
        for (int b = threadIdx.x; b < M; b += blockDim.x) {
            const double ob = (double)(b <= M / 2 ? b : b - M) * delta;
            const double base = 1.0 + (oa * oa + ob * ob) / dof;
            float k1, k2;
            if (dof == 1.0) { k1 = (float)(1.0 / base); k2 = (float)pow(base, -2.0); }
            else { k1 = (float)pow(base, -dof); k2 = (float)pow(base, -dof - 1.0); }
            A[b] = make_float2(k1, k2);
        }
        __syncthreads();
        const float2* R = fft::forward(A, B, plan, tw, threadIdx.x, blockDim.x, BlockSync());
        for (int k = threadIdx.x; k < Mh; k += blockDim.x) {
            const float2 zk = R[k], zm = R[k == 0 ? 0 : M - k];
            Rt[(size_t)k * Pa + a] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            Rt[((size_t)Mhmax + k) * Pa + a] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        }
        __syncthreads();
    }
}

// Column transforms of the row spectra (mirrored to the full torus), real part kept: Kt[kern][k2][k1]
__global__ void __launch_bounds__(kFftThreads) spec_cols_kernel(const GridDesc* __restrict__ gd,
                                                                 const float2* __restrict__ Rt, int Pa, int Mhmax,
                                                                 float* __restrict__ Kt, int Mmax,
                                                                 const float2* __restrict__ tw) {
    if (!gd->spec_dirty) return;
    extern __shared__ float2 sm[];
    const int M = gd->M, Mh = gd->Mh;
    fft::Plan plan;
    fft::make_plan(M, plan);
    float2* A = sm;
    float2* B = sm + M;
    for (int w = blockIdx.x; w < 2 * Mh; w += gridDim.x) {
        const int kern = w / Mh, k = w % Mh;
        const float2* src = Rt + ((size_t)kern * Mhmax + k) * Pa;
        for (int a = threadIdx.x; a < M; a += blockDim.x) A[a] = src[a <= M / 2 ? a : M - a];
        __syncthreads();
        const float2* R = fft::forward(A, B, plan, tw, threadIdx.x, blockDim.x, BlockSync());
        float* dst = Kt + ((size_t)kern * Mhmax + k) * Mmax;
        for (int a = threadIdx.x; a < M; a += blockDim.x) dst[a] = R[a].x;
        __syncthreads();
    }
}

// [k1][k2] (M, Mh) host layout of set_kernels -> transposed Kt[kern][k2][k1]
__global__ void transpose_spectra_kernel(const float* __restrict__ K, float* __restrict__ Kt, int M, int Mh,
                                         int Mmax) {
    __shared__ float tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;   // bx over k2, by over k1
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k1 = by + r, k2 = bx + threadIdx.x;
        if (k1 < M && k2 < Mh) tile[r][threadIdx.x] = K[(size_t)k1 * Mh + k2];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k2 = bx + r, k1 = by + threadIdx.x;
        if (k1 < M && k2 < Mh) Kt[(size_t)k2 * Mmax + k1] = tile[threadIdx.x][r];
    }
}

__global__ void set_grid_kernel(GridDesc* gd, float xmin, float ymin, float width, int n_boxes, int ni, int M) {
    gd->xmin = xmin; gd->ymin = ymin; gd->width = width; gd->inv_width = 1.f / width;
    gd->n_boxes = n_boxes; gd->N = n_boxes * ni; gd->M = M; gd->Mh = M / 2 + 1;
}

int fft_blocks(int work) { return std::max(1, std::min(work, 2 * kNumSMs)); }

size_t fft_smem(int M) { return (size_t)2 * M * sizeof(float2); }

void set_smem_attr(const void* fn, size_t bytes) {
    cudaFuncAttributes a;
    MGB_CUDA(cudaFuncGetAttributes(&a, fn));
    int dev = 0, optin = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    MGB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t mx = std::min(bytes, (size_t)optin - a.sharedSizeBytes);
    MGB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx));
}

template <int NI>
void spread_t(const float2* Y, int64_t n, GridDesc* g, RepBuffers& b, cudaStream_t s) {
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 16 * kNumSMs));
    spread_kernel<NI><<<blocks, 256, 0, s>>>(Y, n, g, b.W.as<float4>(), b.Nmax);
}
template <int NI>
void gather_t(const float2* Y, int64_t n, GridDesc* g, RepBuffers& b, float2* F, cudaStream_t s) {
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 16 * kNumSMs));
    gather_forces_kernel<NI><<<blocks, 256, 0, s>>>(Y, n, g, b.phi.as<float>(), b.Nmax, F);
}

}  // namespace

void rep_set_grid_host(GridDesc* g_dev, float xmin, float ymin, float width, int n_boxes, int ni, int M,
                       cudaStream_t s) {
    set_grid_kernel<<<1, 1, 0, s>>>(g_dev, xmin, ymin, width, n_boxes, ni, M);
    MGB_LAUNCH_CHECK();
}

#define MGB_NI_DISPATCH(ni, F, ...)                 \
    switch (ni) {                                   \
        case 1: F<1>(__VA_ARGS__); break;           \
        case 2: F<2>(__VA_ARGS__); break;           \
        case 3: F<3>(__VA_ARGS__); break;           \
        case 4: F<4>(__VA_ARGS__); break;           \
        case 5: F<5>(__VA_ARGS__); break;           \
        case 6: F<6>(__VA_ARGS__); break;           \
        case 7: F<7>(__VA_ARGS__); break;           \
        default: F<8>(__VA_ARGS__); break;          \
    }

void rep_spread(const float2* Y, int64_t n, GridDesc* g, RepBuffers& b, cudaStream_t s) {
    MGB_NI_DISPATCH(b.ni, spread_t, Y, n, g, b, s);
    MGB_LAUNCH_CHECK();
}

void rep_gather_forces(const float2* Y, int64_t n, GridDesc* g, RepBuffers& b, float2* F, cudaStream_t s) {
    MGB_NI_DISPATCH(b.ni, gather_t, Y, n, g, b, F, s);
    MGB_LAUNCH_CHECK();
}

void ensure_fft_attrs() {
    static thread_local int done_dev = -1;   // per thread: host threads may drive layouts side by side
    int dev = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    if (done_dev == dev) return;
    const size_t mx = fft_smem(fft::kMaxLen);
    set_smem_attr((const void*)row_fwd_kernel, mx);
    set_smem_attr((const void*)row_inv_kernel, mx);
    set_smem_attr((const void*)col_kernel, mx);
    set_smem_attr((const void*)spec_rows_kernel, mx);
    set_smem_attr((const void*)spec_cols_kernel, mx);
    done_dev = dev;
}

void rep_convolve(GridDesc* g, RepBuffers& b, int64_t n, cudaStream_t s, cudaEvent_t* ev) {
    if (b.use3) {
        rep_row_fwd3(g, b, s);
        if (ev) MGB_CUDA(cudaEventRecord(ev[0], s));
        rep_col3(g, b, n, s);
        if (ev) MGB_CUDA(cudaEventRecord(ev[1], s));
        rep_row_inv3(g, b, s);
        if (ev) MGB_CUDA(cudaEventRecord(ev[2], s));
        return;
    }
    const size_t smem = fft_smem(b.Mmax);
    const int pairs = (b.Nmax + 1) / 2;
    row_fwd_kernel<<<fft_blocks(pairs), kFftThreads, smem, s>>>(g, b.W.as<float4>(), b.Nmax, b.WhT.as<float2>(),
                                                                b.Npmax, b.Mhmax, b.tw.as<float2>());
    MGB_LAUNCH_CHECK();
    if (ev) MGB_CUDA(cudaEventRecord(ev[0], s));
    col_kernel<<<fft_blocks(b.Mhmax), kFftThreads, smem, s>>>(g, b.WhT.as<float2>(), b.PhT.as<float2>(), b.Npmax,
                                                              b.Mhmax, b.Kt.as<float>(), b.Mmax, b.tw.as<float2>(),
                                                              b.zpart.as<double>(), n);
    MGB_LAUNCH_CHECK();
    if (ev) MGB_CUDA(cudaEventRecord(ev[1], s));
    row_inv_kernel<<<fft_blocks(pairs), kFftThreads, smem, s>>>(g, b.PhT.as<float2>(), b.Npmax, b.Mhmax,
                                                                b.phi.as<float>(), b.Nmax, b.tw.as<float2>());
    MGB_LAUNCH_CHECK();
    if (ev) MGB_CUDA(cudaEventRecord(ev[2], s));
}

void rep_twiddles(GridDesc* g, RepBuffers& b, cudaStream_t s, bool force) {
    twiddle_kernel<<<fft_blocks(ceil_div(b.Mmax, 256)), 256, 0, s>>>(g, b.tw.as<float2>(), force ? 1 : 0);
    MGB_LAUNCH_CHECK();
}

void rep_prepare_device_spectra(RepBuffers& b) {
    // Rt is only needed by the spectrum generation of the device loop; allocated (and the kernels' shared-memory
    // limits raised) before any stream capture
    const int Pa = b.Mmax / 2 + 1;
    b.Rt.ensure((size_t)2 * b.Mhmax * Pa * sizeof(float2));
    ensure_fft_attrs();
}

void rep_update_spectra(GridDesc* g, RepBuffers& b, float dof, cudaStream_t s) {
    const int Pa = b.Mmax / 2 + 1;
    require(b.Rt.p != nullptr, "rep_prepare_device_spectra must run first");
    const size_t smem = fft_smem(b.Mmax);
    spec_rows_kernel<<<fft_blocks(Pa), kFftThreads, smem, s>>>(g, b.Rt.as<float2>(), Pa, b.Mhmax, b.tw.as<float2>(),
                                                                b.ni, (double)dof);
    MGB_LAUNCH_CHECK();
    spec_cols_kernel<<<fft_blocks(2 * b.Mhmax), kFftThreads, smem, s>>>(g, b.Rt.as<float2>(), Pa, b.Mhmax,
                                                                         b.Kt.as<float>(), b.Mmax, b.tw.as<float2>());
    MGB_LAUNCH_CHECK();
}

void rep_set_spectra_from_host_layout(RepBuffers& b, const float* K1h_dev, const float* K2h_dev, int M,
                                      cudaStream_t s) {
    const int Mh = M / 2 + 1;
    dim3 grid(ceil_div(Mh, 32), ceil_div(M, 32)), block(32, 8);
    transpose_spectra_kernel<<<grid, block, 0, s>>>(K1h_dev, b.Kt.as<float>(), M, Mh, b.Mmax);
    MGB_LAUNCH_CHECK();
    transpose_spectra_kernel<<<grid, block, 0, s>>>(K2h_dev, b.Kt.as<float>() + (size_t)b.Mhmax * b.Mmax, M, Mh,
                                                    b.Mmax);
    MGB_LAUNCH_CHECK();
}

}  // namespace mgb
