// Column pass of the FFT repulsion on the in-place engine (fft3.cuh): src/fftconv.cpp:146-186 (forward column
// transforms, products with the real kernel spectra, inverse column transforms) and the FP64 Z of :226-229.
//
// One work item per (column k of the row half-spectra, channel c), persistent blocks, one shared-memory buffer
// per block (three blocks per SM, so that one block's barriers overlap the others' stages):
//   channels 1 and 2 (x W, y W): forward, times K2, inverse, into outputs 2 and 3;
//   channel 0 (W): forward; sum K1 |W0h|^2 for Z from its spectrum, and its product with K2 into output 1. The
//   reference's potential K1 x W0 (output 0) is never formed: Z comes from the spectrum (Parseval) and the gather
//   reads the potentials 1-3 only.
// The first forward stage reads the live rows (g < N) of WhT from global memory, the last inverse stage writes
// the live rows of PhT, so a column costs 2 (S - 1) shared-memory passes per transform and no reordering pass.
// Output convention as the one-radix engine: PhT = unnormalised inverse (M x the circular convolution).
#include "fftrep.cuh"
#include "fft3.cuh"
#include <vector>
#include <algorithm>

namespace mgb {

namespace {

constexpr int kColThreads = 256;

// transform t of a column pass reads / writes column k of channel a (t = 0) or b (t = 1)
struct ColLoad {
    const float2* a;
    const float2* b;
    __device__ __forceinline__ float2 operator()(int t, int n) const { return (t ? b : a)[n]; }
};
struct ColStore {
    float2* a;
    float2* b;
    __device__ __forceinline__ void operator()(int t, int n, float2 v) const { (t ? b : a)[n] = v; }
};

// last forward stage, product with one real kernel spectrum, first inverse stage (in place), on nbuf buffers
template <int R>
__device__ __noinline__ void middle1(const fft3::Plan& p, float2* __restrict__ A, float2* __restrict__ B, int nbuf,
                                     const float* __restrict__ K) {
    const int pb = p.padR ? R + 1 : R;
    const int nb = p.M / R;
    for (int i = threadIdx.x; i < nb * nbuf; i += blockDim.x) {
        const int t = i >= nb ? 1 : 0;
        const int b = i - t * nb;
        float2* buf = t ? B : A;
        const int base = b * pb;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = buf[base + r];
        fft3::dft_fwd<R>(v);
        const int fb = fft3::base_freq(p, b);
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = fft::cscale(v[q], __ldg(&K[fb + nb * q]));
        fft3::dft_inv<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) buf[base + r] = v[r];
    }
}

// channel 0: the last forward stage, this thread's share of sum K1 |X|^2 (for Z), the product with K2 and the
// first inverse stage (in place in A); returns the share
template <int R>
__device__ __noinline__ double middle2(const fft3::Plan& p, float2* __restrict__ A, const float* __restrict__ K1,
                                       const float* __restrict__ K2) {
    const int pb = p.padR ? R + 1 : R;
    const int nb = p.M / R;
    double zs = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int base = b * pb;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = A[base + r];
        fft3::dft_fwd<R>(v);
        const int fb = fft3::base_freq(p, b);
        float zt = 0.f;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int f = fb + nb * q;
            zt += __ldg(&K1[f]) * (v[q].x * v[q].x + v[q].y * v[q].y);
            v[q] = fft::cscale(v[q], __ldg(&K2[f]));
        }
        zs += (double)zt;
        fft3::dft_inv<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) A[base + r] = v[r];
    }
    return zs;
}

__device__ __forceinline__ double middle2_dispatch(int R, const fft3::Plan& p, float2* A, const float* K1,
                                                   const float* K2) {
    switch (R) {
        case 2: return middle2<2>(p, A, K1, K2);
        case 3: return middle2<3>(p, A, K1, K2);
        case 4: return middle2<4>(p, A, K1, K2);
        case 5: return middle2<5>(p, A, K1, K2);
        case 6: return middle2<6>(p, A, K1, K2);
        case 8: return middle2<8>(p, A, K1, K2);
        case 9: return middle2<9>(p, A, K1, K2);
        case 10: return middle2<10>(p, A, K1, K2);
        case 12: return middle2<12>(p, A, K1, K2);
        case 15: return middle2<15>(p, A, K1, K2);
        case 16: return middle2<16>(p, A, K1, K2);
        case 18: return middle2<18>(p, A, K1, K2);
        default: return middle2<20>(p, A, K1, K2);
    }
}

// One (column, channel) per work item, one shared-memory buffer per block: the three channels' convolutions are
// independent (channel 0 also yields the column's Z share), so a block holds a single transform and the SM
// holds more blocks to overlap one block's barriers with another's stages.
constexpr int kColBlocks = 3;   // 3 x 80 registers x 256 threads; 3 buffers of M = 6000 fit the SM

__global__ void __launch_bounds__(kColThreads, kColBlocks) col3_kernel(GridDesc* __restrict__ gd,
                                                              const fft3::Plan* __restrict__ plans,
                                                              const float2* __restrict__ WhT, float2* __restrict__ PhT,
                                                              int Np, int Mhmax, const float* __restrict__ Kt, int Mmax,
                                                              const float2* __restrict__ tw,
                                                              double* __restrict__ zpart, int64_t n_points) {
    extern __shared__ float2 sm[];
    __shared__ fft3::Plan p;
    __shared__ double red[kColThreads / 32];
    __shared__ int is_last;
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    if (threadIdx.x == 0) p = plans[M];
    __syncthreads();
    float2* A = sm;
    const int S = p.S;
    const int R0 = p.st[0].R, RS = p.st[S - 1].R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int item = blockIdx.x; item < 3 * Mh; item += gridDim.x) {
        // channel 0 first for every column, so that the Z shares are ready early
        const int c = item < Mh ? 0 : (item < 2 * Mh ? 1 : 2);
        const int k = item - c * Mh;
        const float2* src = WhT + ((size_t)c * Mhmax + k) * Np;
        float2* dst = PhT + ((size_t)(c + 1) * Mhmax + k) * Np;
        const float* K1 = Kt + (size_t)k * Mmax;
        const float* K2 = Kt + ((size_t)Mhmax + k) * Mmax;
        MGB_FFT3_RADIX_DISPATCH(R0, fft3::dif_first, p, A, A, 1, ColLoad{src, src}, N, tw);
        __syncthreads();
        for (int s = 1; s < S - 1; ++s) {
            MGB_FFT3_RADIX_DISPATCH(p.st[s].R, fft3::dif_mid, p, s, A, A, 1, tw);
            __syncthreads();
        }
        if (c == 0) {
            double zs = middle2_dispatch(RS, p, A, K1, K2);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) zs += __shfl_xor_sync(0xffffffffu, zs, o);
            if (lane == 0) red[warp] = zs;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
                const bool single = (k == 0) || ((M & 1) == 0 && k == M / 2);
                zpart[k] = single ? t : 2.0 * t;
            }
        } else {
            MGB_FFT3_RADIX_DISPATCH(RS, middle1, p, A, A, 1, K2);
            __syncthreads();
        }
        for (int s = S - 2; s >= 1; --s) {
            MGB_FFT3_RADIX_DISPATCH(p.st[s].R, fft3::dit_mid, p, s, A, A, 1, tw);
            __syncthreads();
        }
        MGB_FFT3_RADIX_DISPATCH(R0, fft3::dit_last, p, A, A, 1, ColStore{dst, dst}, N, tw);
        __syncthreads();
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

// ---------------------------------------------------------------------------------------------- rows
// A block owns 4 grid rows g0..g0+3 (src/fftconv.cpp:129-143 forward, :188-198 inverse). Rows are packed two per
// complex sequence (z = w_g + i w_{g+1}); buffer A holds the pair (g0, g0+1), buffer B the pair (g0+2, g0+3), so
// the transposed spectra of the 4 rows are read and written as 32 contiguous bytes per frequency.
constexpr int kRowThreads = 256;

__device__ __forceinline__ float chan(const float4& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// channel c of rows g0..g0+3 of the charge grid (rows at or past N read as zero)
struct RowLoad {
    const float4* W;
    int pitch, g0, N, c;
    __device__ __forceinline__ float2 operator()(int t, int n) const {
        const int ga = g0 + 2 * t, gb = ga + 1;
        const float x = ga < N ? chan(W[(size_t)ga * pitch + n], c) : 0.f;
        const float y = gb < N ? chan(W[(size_t)gb * pitch + n], c) : 0.f;
        return make_float2(x, y);
    }
};

// potential channel c of rows g0..g0+3: Re to row g0 + 2t, Im to row g0 + 2t + 1, scaled by 1 / M^2
struct PhiStore {
    float* phi;
    size_t plane;
    int pitch, g0, N, c;
    float scale;
    __device__ __forceinline__ void operator()(int t, int n, float2 v) const {
        const int ga = g0 + 2 * t, gb = ga + 1;
        float* base = phi + (size_t)c * plane + n;
        if (ga < N) base[(size_t)ga * pitch] = v.x * scale;
        if (gb < N) base[(size_t)gb * pitch] = v.y * scale;
    }
};

// Forward row transforms of the 3 charge channels, separated into the half spectra of the 4 rows and written
// transposed (WhT[c][k][g]); the consumed rows of W are zeroed for the next spread.
__global__ void __launch_bounds__(kRowThreads, 2) row_fwd3_kernel(const GridDesc* __restrict__ gd,
                                                                  const fft3::Plan* __restrict__ plans,
                                                                  float4* __restrict__ W, int pitchW,
                                                                  float2* __restrict__ WhT, int Np, int Mhmax,
                                                                  const float2* __restrict__ tw) {
    extern __shared__ float2 sm[];
    __shared__ fft3::Plan p;
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    if (threadIdx.x == 0) p = plans[M];
    __syncthreads();
    float2* A = sm;
    float2* B = sm + p.Mp;
    const int S = p.S;
    const int groups = (N + 3) / 4;
    for (int grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const int g0 = 4 * grp;
        const int nbuf = g0 + 2 < N ? 2 : 1;
        for (int c = 0; c < 3; ++c) {
            MGB_FFT3_RADIX_DISPATCH(p.st[0].R, fft3::dif_first, p, A, B, nbuf, RowLoad{W, pitchW, g0, N, c}, N, tw);
            __syncthreads();
            for (int s = 1; s < S; ++s) {
                MGB_FFT3_RADIX_DISPATCH(p.st[s].R, fft3::dif_mid, p, s, A, B, nbuf, tw);
                __syncthreads();
            }
            // rows a, b of a pair from Z_k and Z_{-k}: (Z_k + conj Z_{-k}) / 2 and (Z_k - conj Z_{-k}) / 2i; walked in
            // position order (consecutive threads read consecutive positions), frequencies past M/2 skipped
            for (int pos = threadIdx.x; pos < M; pos += blockDim.x) {
                const int k = fft3::freq_of_pos(p, pos);
                if (k >= Mh) continue;
                const int pk = p.padR ? pos + fft3::udiv(pos, p.mpad) : pos;
                const int pm = fft3::pos_of_freq(p, k == 0 ? 0 : M - k);
                float2* dst = WhT + ((size_t)c * Mhmax + k) * Np + g0;
                for (int t = 0; t < nbuf; ++t) {
                    const float2* buf = t ? B : A;
                    const float2 zk = buf[pk], zm = buf[pm];
                    reinterpret_cast<float4*>(dst)[t] = make_float4(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y),
                                                                    0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
                }
            }
            __syncthreads();
        }
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const int rows = min(4, N - g0);
        for (int i = threadIdx.x; i < rows * N; i += blockDim.x) {
            const int r = i / N, n = i - r * N;
            W[(size_t)(g0 + r) * pitchW + n] = z4;
        }
    }
}

// Inverse row transforms of the potential channels 1-3: each pair rebuilt from the two half spectra (Hermitian
// extension, DC and Nyquist imaginary parts dropped as a c2r does) straight into the digit-reversed positions
// the inverse stages start from, transformed, scaled by 1/M^2 (src/fftconv.cpp:176, 188-198).
__global__ void __launch_bounds__(kRowThreads, 2) row_inv3_kernel(const GridDesc* __restrict__ gd,
                                                                  const fft3::Plan* __restrict__ plans,
                                                                  const float2* __restrict__ PhT, int Np, int Mhmax,
                                                                  float* __restrict__ phi, int pitchP,
                                                                  const float2* __restrict__ tw) {
    extern __shared__ float2 sm[];
    __shared__ fft3::Plan p;
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    if (threadIdx.x == 0) p = plans[M];
    __syncthreads();
    float2* A = sm;
    float2* B = sm + p.Mp;
    const int S = p.S;
    const bool even = (M & 1) == 0;
    const float scale = 1.f / ((float)M * (float)M);
    const size_t plane = (size_t)pitchP * pitchP;
    const int groups = (N + 3) / 4;
    for (int grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const int g0 = 4 * grp;
        const int nbuf = g0 + 2 < N ? 2 : 1;
        for (int c = 1; c < 4; ++c) {   // potentials 1-3 (the gather's); plane 0 is not formed
            // the spectrum enters in position order: consecutive threads write consecutive positions; the loads of
            // the transposed spectra are one 32-byte sector per frequency in either order
#pragma unroll 2
            for (int up = threadIdx.x; up < M; up += blockDim.x) {
                const int k = fft3::freq_of_pos(p, up);
                const int kk = k < Mh ? k : M - k;
                const float4* src = reinterpret_cast<const float4*>(PhT + ((size_t)c * Mhmax + kk) * Np + g0);
                const int pos = p.padR ? up + fft3::udiv(up, p.mpad) : up;
                for (int t = 0; t < nbuf; ++t) {
                    const float4 v = src[t];
                    float2 a = make_float2(v.x, v.y), b = make_float2(v.z, v.w);
                    if (kk == 0 || (even && kk == M / 2)) { a.y = 0.f; b.y = 0.f; }
                    if (k >= Mh) { a.y = -a.y; b.y = -b.y; }
                    (t ? B : A)[pos] = make_float2(a.x - b.y, a.y + b.x);   // a + i b
                }
            }
            __syncthreads();
            for (int s = S - 1; s >= 1; --s) {
                MGB_FFT3_RADIX_DISPATCH(p.st[s].R, fft3::dit_mid, p, s, A, B, nbuf, tw);
                __syncthreads();
            }
            MGB_FFT3_RADIX_DISPATCH(p.st[0].R, fft3::dit_last, p, A, B, nbuf,
                                    PhiStore{phi, plane, pitchP, g0, N, c, scale}, N, tw);
            __syncthreads();
        }
    }
}

size_t col3_smem(int Mp_max) { return (size_t)Mp_max * sizeof(float2); }       // one transform per column block
size_t row3_smem(int Mp_max) { return (size_t)2 * Mp_max * sizeof(float2); }   // two row pairs per row block

}  // namespace

// Plans of every 5-smooth length up to Mmax (table indexed by M; S = 0 where there is none) and the largest
// padded length among them.
void fft3_build_plans(DevBuf& table, int Mmax, int& Mp_max) {
    std::vector<fft3::Plan> plans((size_t)Mmax + 1);
    Mp_max = 0;
    for (int M = 4; M <= Mmax; ++M) {
        if (!fft::is_5smooth(M)) continue;
        if (fft3::make_plan(M, plans[M])) Mp_max = std::max(Mp_max, plans[M].Mp);
    }
    table.ensure(plans.size() * sizeof(fft3::Plan));
    MGB_CUDA(cudaMemcpy(table.p, plans.data(), plans.size() * sizeof(fft3::Plan), cudaMemcpyHostToDevice));
}

// resident blocks of the column kernel for this buffer size (raises its shared-memory limit once per device)
int col3_blocks(int Mp_max) {
    // per thread: host threads may drive layouts side by side
    static thread_local int cached_dev = -1, cached_mp = -1, cached_blocks = 0;
    int dev = 0, optin = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    if (cached_dev == dev && cached_mp == Mp_max) return cached_blocks;
    const size_t smem = col3_smem(Mp_max);
    MGB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes a;
    MGB_CUDA(cudaFuncGetAttributes(&a, (const void*)col3_kernel));
    require(smem + a.sharedSizeBytes <= (size_t)optin, "FFT side too large for the column engine");
    MGB_CUDA(cudaFuncSetAttribute((const void*)col3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, col3_kernel, kColThreads, smem));
    cached_dev = dev;
    cached_mp = Mp_max;
    cached_blocks = std::max(1, per_sm) * kNumSMs;
    return cached_blocks;
}

// resident blocks of a row kernel (raises its shared-memory limit once per device)
int row3_blocks(const void* fn, int Mp_max) {
    const size_t smem = row3_smem(Mp_max);
    int dev = 0, optin = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    MGB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes a;
    MGB_CUDA(cudaFuncGetAttributes(&a, fn));
    require(smem + a.sharedSizeBytes <= (size_t)optin, "FFT side too large for the row engine");
    MGB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kRowThreads, smem));
    return std::max(1, per_sm) * kNumSMs;
}

namespace {
struct RowBlocks {
    int dev = -1, mp = -1, fwd = 0, inv = 0;
};
thread_local RowBlocks g_row_blocks;   // per thread, as the column cache
}  // namespace

// launch sizes of the row kernels (and their shared-memory limits) for this device and buffer size; called when
// the buffers are sized, before any stream capture
void fft3_prepare(int Mp_max) {
    int dev = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    col3_blocks(Mp_max);
    if (g_row_blocks.dev == dev && g_row_blocks.mp == Mp_max) return;
    g_row_blocks.fwd = row3_blocks((const void*)row_fwd3_kernel, Mp_max);
    g_row_blocks.inv = row3_blocks((const void*)row_inv3_kernel, Mp_max);
    g_row_blocks.dev = dev;
    g_row_blocks.mp = Mp_max;
}

void rep_row_fwd3(GridDesc* g, RepBuffers& b, cudaStream_t s) {
    fft3_prepare(b.Mp3max);
    const int blocks = std::min(g_row_blocks.fwd, (b.Nmax + 3) / 4);
    row_fwd3_kernel<<<blocks, kRowThreads, row3_smem(b.Mp3max), s>>>(
        g, b.plans3.as<fft3::Plan>(), b.W.as<float4>(), b.Nmax, b.WhT.as<float2>(), b.Npmax, b.Mhmax,
        b.tw.as<float2>());
    MGB_LAUNCH_CHECK();
}

void rep_row_inv3(GridDesc* g, RepBuffers& b, cudaStream_t s) {
    fft3_prepare(b.Mp3max);
    const int blocks = std::min(g_row_blocks.inv, (b.Nmax + 3) / 4);
    row_inv3_kernel<<<blocks, kRowThreads, row3_smem(b.Mp3max), s>>>(
        g, b.plans3.as<fft3::Plan>(), b.PhT.as<float2>(), b.Npmax, b.Mhmax, b.phi.as<float>(), b.Nmax,
        b.tw.as<float2>());
    MGB_LAUNCH_CHECK();
}

void rep_col3(GridDesc* g, RepBuffers& b, int64_t n, cudaStream_t s) {
    const int blocks = std::min(col3_blocks(b.Mp3max), 3 * b.Mhmax);
    col3_kernel<<<blocks, kColThreads, col3_smem(b.Mp3max), s>>>(
        g, b.plans3.as<fft3::Plan>(), b.WhT.as<float2>(), b.PhT.as<float2>(), b.Npmax, b.Mhmax, b.Kt.as<float>(),
        b.Mmax, b.tw.as<float2>(), b.zpart.as<double>(), n);
    MGB_LAUNCH_CHECK();
}

}  // namespace mgb
